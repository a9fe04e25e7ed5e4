// Batched execution over a shared device block pool: persistent kernels that
// walk a work list of (level descriptor, block) items gathered from many
// cases, plus the per-coarse-step bookkeeping kernels.  Used by the native
// context (native.cu); every case keeps its own descriptors, so a case's
// arithmetic is identical whether it runs alone or in a mix.
#pragma once
#include "bouzidi.cuh"
#include "stream_collide.cuh"
#include "thermal.cuh"

namespace ol {

// Static placement of one (case, level, sub-step) descriptor; the advance
// kernel derives its time-dependent fields from the case clock each step.
struct DescMeta {
  int32_t case_slot;   // index into CaseDev
  int32_t level;       // 1-based level id
  int32_t j;           // sub-step of this level within the coarse step
  int32_t has_parent;
  int32_t ddf;
  int32_t pad;
};

// Per-case device state advanced by the graph itself.
struct CaseDev {
  int64_t t;           // coarse steps completed
  float u_target;
  int32_t ramp_steps;
  int32_t async_depth;
  int32_t status;      // watchdog bits (1 = non-finite density, 2 = density < 0.01)
};

// Pool-wide population / field buffers (A/B = ping-pong by sub-step parity).
struct PoolBufs {
  void *fA, *fB, *gA, *gB;
  float *rhoA, *rhoB, *velA, *velB, *TA, *TB;
};

// Fill the time-dependent fields of every descriptor for coarse step t+1
// (solver_control.jl:19-25 parity, :65-97 sub-steps and temporal weights,
// main.jl:214-218 batched inlet ramp).
__global__ void k_advance(LevelDev *descs, ThermalDev *tdescs, const DescMeta *meta,
                          const CaseDev *cases, PoolBufs P, int n_desc);
// t += 1 for every resident case.
__global__ void k_tick(CaseDev *cases, int n_cases);

// Persistent stream-collide (+ fused thermal DDF) over a work list.
template <int OP, class ST, bool WALE, bool DDF>
__global__ void __launch_bounds__(512, 2)
    k_sc_batched(const LevelDev *__restrict__ descs, const ThermalDev *__restrict__ tdescs,
                 const WorkItem *__restrict__ items, int n_items);

// Batched Bouzidi: one thread per (boundary cell, direction) over the
// concatenated boundary lists of a slot; `f_of_desc` selects f_out (flow)
// or g_out (thermal) of the owning descriptor.
// One cut link of a batched Bouzidi list: its level list and index there.
struct BouzLinkItem {
  int32_t bdesc;
  int32_t link;
};

}  // namespace ol
