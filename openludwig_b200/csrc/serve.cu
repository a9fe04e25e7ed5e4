// Continuous-batching solve service over a native context, behind the C ABI
// so a driver in any language (the reference's Julia main loop through
// ccall) can serve: requests (case descriptors with an arrival time) are
// admitted in arrival order as soon as their device footprint fits the
// context's budget, every resident case advances together (one graph replay
// per coarse step), each case's drag coefficient is evaluated every
// `check_every` of its coarse steps, and a case retires when
// |Cd(t) - Cd(t - window)| < tol (after at least min_steps), when its
// watchdog flags a non-finite density, at max_steps, or when Cd is not
// finite.  The reference runs its cases one after another (run_all_cases,
// main.jl:413-466) and reports time-averaged coefficients
// (surface.jl:58-139); this layer runs many at once.
//
// Times are seconds on the server's steady clock (ol_server_clock), which
// starts when the server is created; latency = finish - arrival.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "coeffs.cuh"
#include "common.cuh"

struct ol_server {
  ol_ctx *ctx = nullptr;
  ol_serve_rule rule{};
  std::chrono::steady_clock::time_point t0;
  struct Req {
    int32_t rid;
    double arrival;
    const ol_case_desc *cd;
    ol_coeff_ref ref;
    size_t need;
  };
  struct Live {
    Req req;
    double admit;
    std::vector<double> cd;
    double coeff[12];
  };
  std::vector<Req> queue;            // submitted, not admitted (arrival order)
  std::map<int32_t, Live> resident;  // by case id
  std::vector<ol_serve_result> done; // retired, not yet polled
  std::map<int32_t, std::vector<double>> history;  // Cd checks of retired requests
  int32_t next_rid = 0;
  std::mutex mu;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

using namespace ol;

extern "C" int ol_server_create(ol_server **out, ol_ctx *ctx, const ol_serve_rule *rule) {
  OL_CHECK_ARG(out && ctx && rule, "ol_server_create: null argument");
  OL_CHECK_ARG(rule->check_every > 0 && rule->window > 0 && rule->window % rule->check_every == 0,
               "ol_server_create: window must be a positive multiple of check_every");
  OL_CHECK_ARG(rule->max_steps > 0 && rule->min_steps >= 0 && rule->tol >= 0.0,
               "ol_server_create: bad max_steps / min_steps / tol");
  ol_server *s = new ol_server();
  s->ctx = ctx;
  s->rule = *rule;
  s->t0 = std::chrono::steady_clock::now();
  *out = s;
  return OL_OK;
}

extern "C" int ol_server_destroy(ol_server *s) {
  if (!s) return OL_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (auto &kv : s->resident) ol_ctx_case_remove(s->ctx, kv.first);
  }
  delete s;
  return OL_OK;
}

extern "C" int ol_server_clock(ol_server *s, double *now_s) {
  OL_CHECK_ARG(s && now_s, "ol_server_clock: null argument");
  *now_s = s->now();
  return OL_OK;
}

extern "C" int ol_serve_submit(ol_server *s, const ol_case_desc *cd, const ol_coeff_ref *ref,
                               double arrival_s, int32_t *rid) {
  OL_CHECK_ARG(s && cd && ref && rid, "ol_serve_submit: null argument");
  size_t need = 0;
  int rc = ol_ctx_case_footprint(s->ctx, cd, &need);
  if (rc) return rc;
  size_t used = 0, budget = 0;
  if ((rc = ol_ctx_stats(s->ctx, &used, &budget, nullptr, nullptr))) return rc;
  if (need > budget)
    return set_error(OL_ERR_NOMEM, "ol_serve_submit: the case needs %zu B, above the budget %zu B",
                     need, budget);
  std::lock_guard<std::mutex> lk(s->mu);
  ol_server::Req r{s->next_rid++, arrival_s, cd, *ref, need};
  auto pos = s->queue.end();
  while (pos != s->queue.begin() && (pos - 1)->arrival > arrival_s) --pos;
  s->queue.insert(pos, r);
  *rid = r.rid;
  return OL_OK;
}

extern "C" int ol_serve_advance(ol_server *s, int32_t *n_resident, int32_t *n_waiting) {
  OL_CHECK_ARG(s, "ol_serve_advance: null server");
  std::lock_guard<std::mutex> lk(s->mu);
  const ol_serve_rule &R = s->rule;
  // admit in arrival order while the footprint fits (the head of the line waits)
  const double t_admit = s->now();
  while (!s->queue.empty() && s->queue.front().arrival <= t_admit) {
    const ol_server::Req r = s->queue.front();
    size_t used = 0, budget = 0;
    int rc = ol_ctx_stats(s->ctx, &used, &budget, nullptr, nullptr);
    if (rc) return rc;
    if (used + r.need > budget) break;
    int32_t cid = -1;
    if ((rc = ol_ctx_case_add(s->ctx, r.cd, &cid))) return rc;
    ol_server::Live lv{r, s->now(), {}, {}};
    s->resident.emplace(cid, lv);
    s->queue.erase(s->queue.begin());
  }
  if (!s->resident.empty()) {
    int rc = ol_ctx_step(s->ctx, R.check_every);
    if (rc == OL_OK) rc = ol_ctx_sync(s->ctx);
    if (rc) return rc;
    std::vector<int32_t> retire;
    for (auto &kv : s->resident) {
      int64_t steps = 0;
      int32_t status = 0;
      if ((rc = ol_ctx_case_info(s->ctx, kv.first, &steps, &status))) return rc;
      ol_server::Live &lv = kv.second;
      if ((rc = ol_ctx_case_coefficients(s->ctx, kv.first, &lv.req.ref, lv.coeff))) return rc;
      const double cd = lv.coeff[0];
      lv.cd.push_back(cd);
      const size_t lag = (size_t)(R.window / R.check_every);
      const bool conv = steps >= R.min_steps && lv.cd.size() > lag &&
                        std::fabs(lv.cd.back() - lv.cd[lv.cd.size() - 1 - lag]) < R.tol;
      if (conv || (status & 1) || steps >= R.max_steps || !std::isfinite(cd)) {
        ol_serve_result res{};
        res.rid = lv.req.rid;
        res.steps = (int32_t)steps;
        res.status = status;
        res.converged = conv ? 1 : 0;
        res.arrival_s = lv.req.arrival;
        res.admit_s = lv.admit;
        res.finish_s = s->now();
        for (int i = 0; i < 12; ++i) res.coeff[i] = lv.coeff[i];
        s->done.push_back(res);
        s->history[lv.req.rid] = lv.cd;
        retire.push_back(kv.first);
      }
    }
    for (int32_t cid : retire) {
      if ((rc = ol_ctx_case_remove(s->ctx, cid))) return rc;
      s->resident.erase(cid);
    }
  }
  if (n_resident) *n_resident = (int32_t)s->resident.size();
  if (n_waiting) *n_waiting = (int32_t)s->queue.size();
  return OL_OK;
}

extern "C" int ol_serve_poll(ol_server *s, ol_serve_result *out, int32_t max, int32_t *n) {
  OL_CHECK_ARG(s && n && max >= 0 && (out || max == 0), "ol_serve_poll: bad argument");
  std::lock_guard<std::mutex> lk(s->mu);
  const int32_t k = std::min<int32_t>(max, (int32_t)s->done.size());
  for (int32_t i = 0; i < k; ++i) out[i] = s->done[i];
  s->done.erase(s->done.begin(), s->done.begin() + k);
  *n = k;
  return OL_OK;
}

extern "C" int ol_serve_history(ol_server *s, int32_t rid, double *cd, int32_t max, int32_t *n) {
  OL_CHECK_ARG(s && n && max >= 0 && (cd || max == 0), "ol_serve_history: bad argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->history.find(rid);
  if (it == s->history.end())
    return set_error(OL_ERR_STATE, "ol_serve_history: request %d has not retired", rid);
  const int32_t k = std::min<int32_t>(max, (int32_t)it->second.size());
  for (int32_t i = 0; i < k; ++i) cd[i] = it->second[i];
  *n = (int32_t)it->second.size();
  return OL_OK;
}
