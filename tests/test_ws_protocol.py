"""The producer / consumer protocol of the warp-specialised kernels (k_sc_ws
in ws.cuh, k_thermal_ws in thermal_ws.cuh), model-checked on the CPU.

The model follows the kernels' order of operations, one step at a time, and
runs it under random interleavings of one producer warp and three consumer
warps:

* producer: publish the descriptors (neighbour row, block id) of blocks 0
  and 1; then for each block j: publish block j+1's descriptors (j >= 1),
  wait until every consumer has released block j - B (B stage buffers), and
  issue block j's copies into buffer j % B (the "landed" barrier of j);
* consumer: wait for block j to land, barrier, read block j's descriptors
  (spread), barrier, pull, release block j, load block j+1's out-of-block
  values (its descriptors), update block j (its descriptors again: the
  output address).

Checked on every step: descriptors are written only into ring slots no
consumer still reads, and a block's copies go only into a buffer no consumer
still pulls from; each read finds the descriptors of the block it wants.
The ring sizes and buffer counts are read from the kernel headers.  The
model finds the race of a double-buffered stage with a 4-slot ring: the
producer's look-ahead then overwrites the descriptors of a block a slow
consumer is still updating."""
import random
import re
from pathlib import Path

import pytest

CSRC = Path(__file__).resolve().parents[1] / "openludwig_b200" / "csrc"


def _const(path: Path, name: str) -> str:
    m = re.search(rf"constexpr int {name} = ([^;]+);", path.read_text())
    assert m, (path, name)
    return m.group(1).strip()


def _params():
    ws_ring = int(_const(CSRC / "ws.cuh", "kWsRing"))
    tw_ring = int(_const(CSRC / "thermal_ws.cuh", "kTwRing"))
    tw_tab = _const(CSRC / "thermal_ws.cuh", "kTwTab")
    m = re.fullmatch(r"(\d+) \* kTwBuf", tw_tab)
    assert m, tw_tab
    return {"k_sc_ws": (1, ws_ring), "k_thermal_ws": (int(m.group(1)), tw_ring)}


class Violation(AssertionError):
    pass


def _run(buffers: int, ring: int, cnt: int, n_cons: int, rng: random.Random) -> None:
    slot = [None] * ring                 # block whose descriptors a slot holds
    landed = [False] * cnt
    released = [0] * cnt                 # consumers that released block j
    using = [set() for _ in range(n_cons)]    # blocks whose descriptors a consumer reads
    pulling = [None] * n_cons            # block a consumer may still pull from its buffer
    bar_count = {}                       # (barrier id, block) -> consumers arrived

    def publish(p):
        for c in range(n_cons):
            for i in using[c]:
                if i != p and i % ring == p % ring:
                    raise Violation(f"descriptors of {p} overwrite those of {i} in use")
        slot[p % ring] = p

    def read(c, p):
        if slot[p % ring] != p:
            raise Violation(f"consumer {c} reads {slot[p % ring]} instead of {p}")

    def producer():
        publish(0)
        yield
        if cnt > 1:
            publish(1)
            yield
        for j in range(cnt):
            if 1 <= j and j + 1 < cnt:
                publish(j + 1)
                yield
            if j >= buffers:
                while released[j - buffers] < n_cons:
                    yield
            for c in range(n_cons):
                i = pulling[c]
                if i is not None and i != j and i % buffers == j % buffers:
                    raise Violation(f"copies of {j} overwrite buffer of {i}")
            landed[j] = True
            yield

    def barrier(key):
        bar_count[key] = bar_count.get(key, 0) + 1
        while bar_count[key] < n_cons:
            yield

    def consumer(c):
        for j in range(cnt):
            while not landed[j]:
                yield
            pulling[c] = j
            yield from barrier((1, j))
            using[c].add(j)
            read(c, j)                      # spread: neighbour row, ghost row
            yield
            yield from barrier((2, j))
            yield                           # pull
            pulling[c] = None
            released[j] += 1
            yield
            if j + 1 < cnt:
                using[c].add(j + 1)
                read(c, j + 1)              # out-of-block values of block j+1
                yield
                using[c].discard(j + 1)
            for _ in range(rng.randrange(1, 8)):   # the update, of varying length
                read(c, j)
                yield
            using[c].discard(j)

    actors = [producer()] + [consumer(c) for c in range(n_cons)]
    live = list(range(len(actors)))
    while live:
        a = rng.choice(live)
        try:
            next(actors[a])
        except StopIteration:
            live.remove(a)


@pytest.mark.parametrize("kernel", ["k_sc_ws", "k_thermal_ws"])
def test_protocol_never_overwrites_what_a_consumer_uses(kernel):
    buffers, ring = _params()[kernel]
    rng = random.Random(20261203)
    for _ in range(400):
        _run(buffers, ring, cnt=rng.randrange(1, 14), n_cons=3, rng=rng)


@pytest.mark.parametrize("buffers,ring", [(2, 4), (1, 3)])
def test_model_finds_the_race_of_a_short_ring(buffers, ring):
    """Too few descriptor slots for the look-ahead: two stage buffers with
    four slots, or one with three.  Some interleaving lets the producer
    overwrite a slot that a consumer still reads."""
    rng = random.Random(7)
    found = False
    for _ in range(400):
        try:
            _run(buffers, ring, cnt=12, n_cons=3, rng=rng)
        except Violation:
            found = True
            break
    assert found
