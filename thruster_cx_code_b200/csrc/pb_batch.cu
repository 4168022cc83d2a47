// Batched stepping of several simulators on one GPU (included by pb_runtime.cu).
//
// The reference advances one aperture simulation per process and runs sweeps as one
// process per sweep point (Python/benchmarks/benchmark_perveance.py:78-164).  Here many
// instances share the device: each keeps its particles, fields and multigrid hierarchy
// resident and its particle kernels run on its own stream, so the kernels of different
// instances overlap.  Their field solves, which are latency-bound on one grid, run as one
// cooperative launch in which every instance gets a contiguous range of blocks with its
// own grid barrier and reductions (k_poisson_batch).

#include <condition_variable>
#include <queue>
#include <thread>

// Host threads that enqueue the members' step halves in parallel (the streams form): a
// persistent pool; run(f) calls f(w) on every worker w and on the calling thread (the last
// index) and returns when all are done.
struct EnqueuePool {
  std::vector<std::thread> th;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::function<void(int)> task;
  long long generation = 0;
  int pending = 0;
  bool stop = false;
  int workers() const { return (int)th.size(); }
  void start(int n) {
    for (int w = 0; w < n; ++w)
      th.emplace_back([this, w] {
        long long seen = 0;
        while (true) {
          std::function<void(int)> f;
          {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return stop || generation != seen; });
            if (stop) return;
            seen = generation;
            f = task;
          }
          f(w);
          std::lock_guard<std::mutex> lk(mu);
          if (--pending == 0) cv_done.notify_one();
        }
      });
  }
  void run(const std::function<void(int)>& f) {
    {
      std::lock_guard<std::mutex> lk(mu);
      task = f;
      pending = (int)th.size();
      ++generation;
    }
    cv_work.notify_all();
    f((int)th.size());
    std::unique_lock<std::mutex> lk(mu);
    cv_done.wait(lk, [&] { return pending == 0; });
  }
  ~EnqueuePool() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv_work.notify_all();
    for (auto& t : th) t.join();
  }
};

struct pb_batch {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  PoissonArgs* dargs = nullptr;  // device copy of every field-solve argument block of a run
  PoissonArgs* hargs = nullptr;  // pinned staging
  size_t args_cap = 0, dargs_cap = 0;
  MgRebuildArgs* dmg = nullptr;  // the hierarchy-rebuild argument blocks, one beside each of the above
  MgRebuildArgs* hmg = nullptr;
  size_t mg_cap = 0, dmg_cap = 0;
  int* dblk = nullptr;           // block -> argument-block maps of every launch of a run
  int* hblk = nullptr;
  size_t blk_cap = 0, dblk_cap = 0;
  pb_step_report* hrep = nullptr;  // pinned per-step reports
  size_t rep_cap = 0;
  std::vector<cudaEvent_t> ev_inst;  // per instance: "pre-solve half enqueued" / "stream done"
  std::vector<cudaEvent_t> ev_solve; // per launch of a step
  double last_ms = 0.0;
  double last_host_ms = 0.0;   // host time spent enqueuing the last run (ev0 to the last enqueue)
  double last_solve_ms = 0.0;  // device time of the field-solve launches of the last run (streams form)
  std::vector<cudaEvent_t> tev; // timing events around the solve launches
  long long launches = 0;
  // CUDA graphs of whole batch steps (pb_batch_set_graphs): one graph per step shape of the
  // set (each member's step parameters without the step number and its state signature)
  int graphs_on = 0, graphs_broken = 0;
  std::string graph_error;
  struct StepGraph {
    uint64_t key = 0;
    cudaGraphExec_t exec = nullptr;
    PoissonArgs* dargs = nullptr;     // the step's field-solve argument blocks, owned by the graph
    MgRebuildArgs* dmg = nullptr;     // and the hierarchy-rebuild blocks beside them
    int* dblk = nullptr;
    pb_step_report** dreps = nullptr; // the members' report buffers, gathered at the end of the step
    std::vector<long long> launches;  // kernels of each member in the step
    long long own_launches = 0;       // the step's field solves and report gather
  };
  std::vector<StepGraph> graphs;
  pb_step_report* ring = nullptr;     // reports of a run, [step][member]
  pb_step_report* hring = nullptr;
  size_t ring_cap = 0;
  int* slot = nullptr;                // next ring row
  cudaEvent_t ev_fork = nullptr;
  long long graph_captures = 0, graph_replays = 0;
  // host threads of the streams form (created on first use); one by default: more measured
  // slower (64 sweep points: 3.6 ms of host time per step on one thread, 6.7 ms on eight,
  // and 5% more device time), the driver serialises the launches anyway
  int enqueue_threads = 1;  // total, the calling thread included (0: chosen from the host)
  std::unique_ptr<EnqueuePool> pool;
};

namespace {

struct SolveLaunch {
  int step;
  std::vector<int> inst;  // instances (indices into the run's simulator list)
  size_t args_off;        // first argument block
  size_t blk_off;         // first entry of the block map
  size_t map_len;         // entries of the block map: an offset per block, then per block its
                          // instance count and instances
  int nblocks;
  size_t smem;
};

// After a batch run: block-ns per field-solve launch of the run's solves (their counters
// were cleared at its start).  The estimate moves only when the run's figure is off by more
// than 30%, so that the block shares, and the step graphs captured with them, stay put while
// the cost does.
static int32_t measure_solve(Sim* s) {
  unsigned long long ns[2] = {0, 0};
  CK(cudaMemcpy(ns, s->solve_ns, sizeof(ns), cudaMemcpyDeviceToHost));
  if (ns[1] == 0) return PB_OK;
  const double w = (double)ns[0] / (double)ns[1];
  if (!(s->solve_work > 0.0) || w > 1.3 * s->solve_work || w * 1.3 < s->solve_work) s->solve_work = w;
  return PB_OK;
}

// Work of one field-solve launch of each instance, for its block share: the block-ns its
// solves took in the last batch run it was part of (quantised to steps of 2^(1/4), so that
// the shares, and with them the captured step graphs, change only when the cost does), or,
// for an instance not yet measured, its node count times the median block-ns per node of
// the measured ones (its node count alone when none is measured).
std::vector<long> solve_work(pb_sim* const* sims, const std::vector<int>& inst) {
  std::vector<double> ratio;
  for (int i : inst) {
    const Sim* s = &sims[i]->s;
    if (s->solve_work > 0.0) ratio.push_back(s->solve_work / ((double)s->ny * s->nx));
  }
  double med = 0.0;
  if (!ratio.empty()) {
    std::sort(ratio.begin(), ratio.end());
    med = ratio[ratio.size() / 2];
  }
  std::vector<long> work;
  for (int i : inst) {
    const Sim* s = &sims[i]->s;
    const double nodes = (double)s->ny * s->nx;
    double w = s->solve_work > 0.0 ? s->solve_work : (med > 0.0 ? med * nodes : nodes);
    if (med > 0.0 || s->solve_work > 0.0) w = std::exp2(std::round(4.0 * std::log2(std::max(w, 1.0))) / 4.0);
    work.push_back((long)std::min(w, 1e15));
  }
  return work;
}

// Blocks of one launch shared out by each instance's cost (solve_work): the smallest makespan
// T (found by bisection) for which the instances costing more than T get ceil(cost / T) blocks
// of their own and the others fit, first fit by decreasing cost, into blocks of capacity T that
// run them one after another; the blocks left over go one at a time to the instance, alone on
// its blocks, with the largest cost per block.  Packing the cheap instances frees blocks that
// one block each would tie up.  Returns per block the instances (indices into work) it runs,
// an instance's own blocks consecutive.
std::vector<std::vector<int>> plan_blocks(const std::vector<long>& work, int total) {
  const int m = (int)work.size();
  auto pack = [&](double T, std::vector<int>* own, std::vector<std::vector<int>>* bins) -> int {
    int need = 0;
    std::vector<int> small;
    for (int i = 0; i < m; ++i) {
      if ((double)work[i] > T) {
        const int k = (int)std::ceil((double)work[i] / T);
        need += k;
        if (own) (*own)[i] = k;
      } else {
        small.push_back(i);
      }
    }
    std::stable_sort(small.begin(), small.end(), [&](int a, int b) { return work[a] > work[b]; });
    std::vector<double> load;
    std::vector<std::vector<int>> bl;
    for (int i : small) {
      size_t k = 0;
      while (k < load.size() && load[k] + (double)work[i] > T) ++k;
      if (k == load.size()) { load.push_back(0.0); bl.emplace_back(); }
      load[k] += (double)work[i];
      bl[k].push_back(i);
    }
    if (bins) *bins = bl;
    return need + (int)bl.size();
  };
  double sum = 0.0, mx = 0.0;
  for (long w : work) { sum += (double)w; mx = std::max(mx, (double)w); }
  double lo = sum / total, hi = std::max(mx, lo);
  for (int it = 0; it < 64 && hi > lo * (1.0 + 1e-9); ++it) {
    const double mid = 0.5 * (lo + hi);
    if (pack(mid, nullptr, nullptr) <= total) hi = mid; else lo = mid;
  }
  std::vector<int> own(m, 0);
  std::vector<std::vector<int>> bins;
  int used = pack(hi, &own, &bins);
  // an instance alone in its block takes further blocks like one with blocks of its own
  std::vector<std::vector<int>> shared;
  for (auto& b : bins) {
    if (b.size() == 1) own[b[0]] = 1;
    else shared.push_back(b);
  }
  using E = std::pair<double, int>;
  auto lower = [](const E& a, const E& b) { return a.first < b.first || (a.first == b.first && a.second > b.second); };
  std::priority_queue<E, std::vector<E>, decltype(lower)> q(lower);
  for (int i = 0; i < m; ++i)
    if (own[i] > 0) q.push({(double)work[i] / own[i], i});
  for (; used < total && !q.empty(); ++used) {
    const int i = q.top().second;
    q.pop();
    own[i] += 1;
    q.push({(double)work[i] / own[i], i});
  }
  std::vector<std::vector<int>> blocks;
  for (int i = 0; i < m; ++i)
    for (int k = 0; k < own[i]; ++k) blocks.push_back({i});
  for (auto& b : shared) blocks.push_back(b);
  while ((int)blocks.size() < total) blocks.emplace_back();
  return blocks;
}

// Device memory held by one simulator (an estimate from its capacities, for admission).
int64_t sim_device_bytes(const Sim* s) {
  const int64_t N = (int64_t)s->ny * s->nx;
  int64_t b = 0;
  for (int k = 0; k < 2; ++k) b += 2LL * s->sp[k].cap * (5 * 4 + 4 + (s->sp[k].ion ? 1 : 0));
  b += N * (9 * 8 + 9 * 4 + 32 + 4 + 2 + 3 * 4);  // double and float fields, E corners, masks, count maps
  for (size_t l = 0; l < s->lev.size(); ++l) {
    const int64_t Nl = (int64_t)s->lev[l].ny * s->lev[l].nx;
    b += Nl * 4 * (1 + (l ? 2 : 0));  // dinv; r and z below the fine level
    b += Nl * 4 * ((s->lev[l].R ? 25 : 0) + (s->lev[l].U ? 18 : 0));
  }
  b += (int64_t)s->ncap * s->ncap * (4 + 8);  // coarsest inverse and the rebuild's dense scratch
  b += (int64_t)s->ncap * MG_PANEL * 4 * 8;
  for (size_t l = 1; l < s->lev.size(); ++l) b += (int64_t)s->lev[l].ny * s->lev[l].nx * (1 + 9 * 4);
  b += 4LL * (int64_t)s->sort_cap * 4 + (int64_t)s->hist_cap * 4 + 2LL * (int64_t)s->tile_cap * 8;
  b += (int64_t)s->see_cap * 16 + (int64_t)s->angle_cap * 8;
  return b;
}

__global__ void k_batch_reports(pb_step_report* const* src, int n, pb_step_report* ring, int* slot) {
  const int row = *slot;
  constexpr int W = (int)(sizeof(pb_step_report) / 4);
  for (int t = threadIdx.x; t < n * W; t += blockDim.x) {
    const int i = t / W, w = t - i * W;
    reinterpret_cast<uint32_t*>(ring + (size_t)row * n + i)[w] = reinterpret_cast<const uint32_t*>(src[i])[w];
  }
  __syncthreads();
  if (threadIdx.x == 0) *slot = row + 1;
}

void free_batch_graphs(pb_batch* b) {
  for (auto& g : b->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.dargs) cudaFree(g.dargs);
    if (g.dmg) cudaFree(g.dmg);
    if (g.dblk) cudaFree(g.dblk);
    if (g.dreps) cudaFree(g.dreps);
  }
  b->graphs.clear();
}

template <class T>
int32_t grow_pinned(T** p, size_t* cap, size_t need) {
  if (need <= *cap) return PB_OK;
  if (*p) CK(cudaFreeHost(*p));
  *p = nullptr;
  *cap = 0;
  CK(cudaMallocHost((void**)p, need * sizeof(T)));
  *cap = need;
  return PB_OK;
}

}  // namespace

// The hierarchy rebuild of the instances of one solve launch, on the launch's blocks, before
// their field solve (when any of them has had sputter breaks; a clean instance returns at once).
static int32_t launch_mg_rebuild_batch(pb_batch* b, pb_sim* const* sims, const SolveLaunch& L,
                                       const MgRebuildArgs* dm, const int* db, bool capturing) {
  bool any = false;
  for (int i : L.inst) any = any || sims[i]->s.erosion_seen;
  if (!any) return PB_OK;
  void* kargs[] = {(void*)&dm, (void*)&db};
  if (capturing) {
    CK(cudaLaunchCooperativeKernel((void*)k_mg_rebuild_batch, dim3(L.nblocks), dim3(PT), kargs, 0, b->stream));
  } else if (int32_t rc = coop_launch(b->device, b->stream, [&]() {
               return cudaLaunchCooperativeKernel((void*)k_mg_rebuild_batch, dim3(L.nblocks), dim3(PT), kargs, 0,
                                                  b->stream);
             })) {
    return rc;
  }
  ++b->launches;
  return PB_OK;
}

// ------------------------------------------------------------------ batch steps as graphs
// One step of every member: fork from the batch stream, the pre-solve halves on the members'
// streams, the step's cooperative field-solve launches on the batch stream, the post-solve
// halves, then the members' report buffers gathered into row `slot` of the ring.  Enqueued
// into a graph while the members are in capture mode (the Philox step keys then come from
// each member's step_dev, which the captured step advances), or directly otherwise.
static int32_t enqueue_batch_step(pb_batch* b, pb_sim* const* sims, int n, const pb_step_params* const* P,
                                  const std::vector<const SolveLaunch*>& Ls, const PoissonArgs* dargs,
                                  const MgRebuildArgs* dmg, const int* dblk, size_t args0, size_t blk0,
                                  pb_step_report** dreps, bool capturing, std::vector<long long>* launches) {
  int32_t rc;
  CK(cudaEventRecord(b->ev_fork, b->stream));
  for (int i = 0; i < n; ++i) CK(cudaStreamWaitEvent(sims[i]->s.stream, b->ev_fork, 0));
  std::vector<long long> l0(n);
  for (int i = 0; i < n; ++i) {
    l0[i] = sims[i]->s.launches;
    if ((rc = enqueue_step_pre(sims[i], P[i]))) return rc;
    CK(cudaEventRecord(b->ev_inst[i], sims[i]->s.stream));
  }
  std::vector<int> solved_by(n, -1);
  for (size_t li = 0; li < Ls.size(); ++li) {
    const SolveLaunch& L = *Ls[li];
    for (int i : L.inst) {
      CK(cudaStreamWaitEvent(b->stream, b->ev_inst[i], 0));
      solved_by[i] = (int)li;
    }
    const PoissonArgs* da = dargs + (L.args_off - args0);
    const int* db = dblk + (L.blk_off - blk0);
    if ((rc = launch_mg_rebuild_batch(b, sims, L, dmg + (L.args_off - args0), db, capturing))) return rc;
    void* kargs[] = {(void*)&da, (void*)&db};
    if (capturing) {
      CK(cudaLaunchCooperativeKernel((void*)k_poisson_batch, dim3(L.nblocks), dim3(PT), kargs, L.smem, b->stream));
    } else if ((rc = coop_launch(b->device, b->stream, [&]() {
                  return cudaLaunchCooperativeKernel((void*)k_poisson_batch, dim3(L.nblocks), dim3(PT), kargs, L.smem,
                                                     b->stream);
                }))) {
      return rc;
    }
    ++b->launches;
    CK(cudaEventRecord(b->ev_solve[li], b->stream));
  }
  for (int i = 0; i < n; ++i) {
    Sim* s = &sims[i]->s;
    if (solved_by[i] >= 0) CK(cudaStreamWaitEvent(s->stream, b->ev_solve[solved_by[i]], 0));
    if ((rc = enqueue_step_post(sims[i], P[i]))) return rc;
    if (capturing) {
      k_step_advance<<<1, 1, 0, s->stream>>>(s->step_dev);
      CK(cudaGetLastError());
      ++s->launches;
    }
    CK(cudaEventRecord(b->ev_inst[i], s->stream));
    CK(cudaStreamWaitEvent(b->stream, b->ev_inst[i], 0));
    if (launches) (*launches)[i] = s->launches - l0[i];
  }
  k_batch_reports<<<1, 256, 0, b->stream>>>(dreps, n, b->ring, b->slot);
  CK(cudaGetLastError());
  ++b->launches;
  return PB_OK;
}

template <class T>
static cudaError_t dcopy(T** dst, const T* src, size_t n) {
  *dst = nullptr;
  cudaError_t e = cudaMalloc((void**)dst, std::max<size_t>(n, 1) * sizeof(T));
  if (e == cudaSuccess && n) e = cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

// pb_batch_run with graphs: each step's shape is captured once and replayed; a step that
// cannot be captured is enqueued directly (and graphs stay off for the batch).
static int32_t batch_run_graphs(pb_batch* b, pb_sim* const* sims, int n, const pb_step_params* params, int K,
                                const std::vector<SolveLaunch>& plan) {
  int32_t rc = PB_OK;
  std::vector<pb_step_report*> reps(n);
  for (int i = 0; i < n; ++i) reps[i] = sims[i]->s.rep_dev;
  pb_step_report** dreps_run = nullptr;
  CK(dcopy(&dreps_run, reps.data(), (size_t)n));
  size_t pi = 0;
  for (int k = 0; k < K && rc == PB_OK; ++k) {
    std::vector<const pb_step_params*> P(n);
    for (int i = 0; i < n; ++i) P[i] = &params[(size_t)i * K + k];
    std::vector<const SolveLaunch*> Ls;
    for (; pi < plan.size() && plan[pi].step == k; ++pi) Ls.push_back(&plan[pi]);
    const size_t args0 = Ls.empty() ? 0 : Ls.front()->args_off, blk0 = Ls.empty() ? 0 : Ls.front()->blk_off;
    size_t nargs = 0, nblk = 0;
    for (const SolveLaunch* L : Ls) { nargs += L->inst.size(); nblk += L->map_len; }
    uint64_t key = fnv_v(1469598103934665603ull, n);
    for (int i = 0; i < n; ++i) {
      key = fnv_v(key, sims[i]);
      key = fnv_v(key, params_digest(P[i]));
      key = fnv_v(key, state_signature(sims[i]));
    }
    key = fnv(key, b->hblk + blk0, nblk * sizeof(int));  // the step's block shares
    pb_batch::StepGraph* g = nullptr;
    for (auto& e : b->graphs)
      if (e.key == key) g = &e;
    // the members' step keys as the step expects them (they advance inside a replayed graph)
    for (int i = 0; i < n; ++i) {
      Sim* s = &sims[i]->s;
      if ((long long)(uint32_t)P[i]->iteration != s->step_dev_val) {
        k_step_set<<<1, 1, 0, b->stream>>>(s->step_dev, (uint32_t)P[i]->iteration);
        CK(cudaGetLastError());
      }
    }
    if (g) {
      for (int i = 0; i < n; ++i) {
        Sim* s = &sims[i]->s;
        const int flips = 1 + (P[i]->sort_now ? 1 : 0);
        for (int sp = 0; sp < 2; ++sp) s->sp[sp].cur ^= (flips & 1);
        s->counts_valid = true;
        s->sp_dx = P[i]->dx;
        s->sp_dy = P[i]->dy;
        if (P[i]->erosion_on) s->erosion_seen = true;
        s->launches += g->launches[i];
      }
      CK(cudaGraphLaunch(g->exec, b->stream));
      b->launches += g->own_launches;
      ++b->graph_replays;
    } else if (!b->graphs_broken) {
      pb_batch::StepGraph ng;
      ng.key = key;
      ng.launches.assign(n, 0);
      CK(dcopy(&ng.dargs, b->hargs + args0, nargs));
      CK(dcopy(&ng.dmg, b->hmg + args0, nargs));
      CK(dcopy(&ng.dblk, b->hblk + blk0, nblk));
      CK(dcopy(&ng.dreps, reps.data(), (size_t)n));
      // host state of the members, restored if the step cannot be captured
      std::vector<std::array<double, 7>> saved(n);
      for (int i = 0; i < n; ++i) {
        const Sim* s = &sims[i]->s;
        saved[i] = {(double)s->sp[0].cur, (double)s->sp[1].cur, (double)s->counts_valid, s->sp_dx, s->sp_dy,
                    (double)s->launches, (double)s->erosion_seen};
      }
      const long long bl0 = b->launches;
      cudaError_t ce = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
      int32_t crc = ce == cudaSuccess ? PB_OK : PB_ERR_CUDA;
      if (crc == PB_OK) {
        for (int i = 0; i < n; ++i) sims[i]->s.capturing = 1;
        crc = enqueue_batch_step(b, sims, n, P.data(), Ls, ng.dargs, ng.dmg, ng.dblk, args0, blk0, ng.dreps, true,
                                 &ng.launches);
        for (int i = 0; i < n; ++i) sims[i]->s.capturing = 0;
        cudaGraph_t graph = nullptr;
        ce = cudaStreamEndCapture(b->stream, &graph);
        if (crc == PB_OK && ce == cudaSuccess && graph) ce = cudaGraphInstantiate(&ng.exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (ce != cudaSuccess || !ng.exec) crc = crc ? crc : PB_ERR_CUDA;
      }
      if (crc != PB_OK) {
        b->graphs_broken = 1;
        b->graph_error = crc == PB_ERR_CUDA && ce != cudaSuccess ? std::string("batch step capture: ") +
                                                                       cudaGetErrorString(ce)
                                                                 : g_err;
        cudaGetLastError();
        for (int i = 0; i < n; ++i) {
          Sim* s = &sims[i]->s;
          s->sp[0].cur = (int)saved[i][0]; s->sp[1].cur = (int)saved[i][1];
          s->counts_valid = saved[i][2] != 0.0; s->sp_dx = saved[i][3]; s->sp_dy = saved[i][4];
          s->launches = (long long)saved[i][5];
          s->erosion_seen = saved[i][6] != 0.0;
        }
        b->launches = bl0;
        if (ng.exec) cudaGraphExecDestroy(ng.exec);
        cudaFree(ng.dargs); cudaFree(ng.dmg); cudaFree(ng.dblk); cudaFree(ng.dreps);
      } else {
        if (b->graphs.size() >= 16) free_batch_graphs(b);
        ng.own_launches = b->launches - bl0;
        b->graphs.push_back(ng);
        CK(cudaGraphLaunch(ng.exec, b->stream));
        ++b->graph_captures;
      }
    }
    if (b->graphs_broken && !g) {
      // enqueue this step directly (arguments from the run's device copy)
      for (int i = 0; i < n; ++i) sims[i]->s.step_dev_val = -1;
      if ((rc = enqueue_batch_step(b, sims, n, P.data(), Ls, b->dargs, b->dmg, b->dblk, 0, 0, dreps_run, false,
                                   nullptr))) {
        cudaFree(dreps_run);
        return rc;
      }
      continue;
    }
    for (int i = 0; i < n; ++i) sims[i]->s.step_dev_val = (long long)(uint32_t)P[i]->iteration + 1;
  }
  cudaFree(dreps_run);
  return PB_OK;
}

extern "C" {

int32_t pb_batch_create(pb_batch** out, int32_t device) {
  if (!out) return fail(PB_ERR_ARG, "pb_batch_create: null output");
  pb_batch* b = new pb_batch();
  b->device = device;
  CK(cudaSetDevice(device));
  CK(cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device));
  CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&b->ev0));
  CK(cudaEventCreate(&b->ev1));
  CK(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
  CK(cudaMalloc((void**)&b->slot, sizeof(int)));
  CK(cudaFuncSetAttribute((const void*)k_poisson_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)mg_solve_smem_bytes(MG_MAX_COARSE, b->num_sms, 1)));
  CK(cudaFuncSetAttribute((const void*)k_poisson_batch, cudaFuncAttributePreferredSharedMemoryCarveout,
                          (int)cudaSharedmemCarveoutMaxL1));
  *out = b;
  return PB_OK;
}

int32_t pb_batch_destroy(pb_batch* b) {
  if (!b) return PB_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->dargs) cudaFree(b->dargs);
  if (b->dmg) cudaFree(b->dmg);
  if (b->dblk) cudaFree(b->dblk);
  if (b->hargs) cudaFreeHost(b->hargs);
  if (b->hmg) cudaFreeHost(b->hmg);
  if (b->hblk) cudaFreeHost(b->hblk);
  if (b->hrep) cudaFreeHost(b->hrep);
  free_batch_graphs(b);
  if (b->ring) cudaFree(b->ring);
  if (b->hring) cudaFreeHost(b->hring);
  if (b->slot) cudaFree(b->slot);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  for (cudaEvent_t e : b->tev) cudaEventDestroy(e);
  for (cudaEvent_t e : b->ev_inst) cudaEventDestroy(e);
  for (cudaEvent_t e : b->ev_solve) cudaEventDestroy(e);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return PB_OK;
}

int32_t pb_batch_run(pb_batch* b, pb_sim* const* sims, int32_t n, const pb_step_params* params, int32_t K,
                     pb_step_report* reports) {
  if (!b || !sims || n <= 0 || K <= 0 || !params) return fail(PB_ERR_ARG, "pb_batch_run: bad arguments");
  CK(cudaSetDevice(b->device));
  int32_t rc;
  for (int i = 0; i < n; ++i) {
    Sim* s = &sims[i]->s;
    if (!s->domain_set) return fail(PB_ERR_STATE, "pb_batch_run: simulator " + std::to_string(i) + " has no domain");
    if (s->device != b->device) return fail(PB_ERR_ARG, "pb_batch_run: simulators must be on the batch's device");
    for (int j = 0; j < i; ++j)
      if (sims[j] == sims[i]) return fail(PB_ERR_ARG, "pb_batch_run: a simulator appears twice");
    for (int k = 0; k < K; ++k)
      if (params[(size_t)i * K + k].rf_grid >= 0)
        return fail(PB_ERR_ARG, "pb_batch_run: RF co-extraction steps (a second field solve inside the step) run "
                                "with pb_sim_run, not in a batch");
    if ((rc = ensure_room(s, &params[(size_t)i * K], K))) return rc;
  }
  // ---- plan the field-solve launches of the whole run
  std::vector<SolveLaunch> plan;
  size_t nargs = 0, nblk = 0;
  for (int k = 0; k < K; ++k) {
    std::vector<int> need;
    for (int i = 0; i < n; ++i) {
      const pb_step_params& p = params[(size_t)i * K + k];
      if (p.do_poisson && p.picard_iters > 0) need.push_back(i);
    }
    for (size_t c0 = 0; c0 < need.size(); c0 += (size_t)b->num_sms) {
      SolveLaunch L;
      L.step = k;
      L.inst.assign(need.begin() + c0, need.begin() + std::min(need.size(), c0 + (size_t)b->num_sms));
      L.args_off = nargs;
      L.blk_off = nblk;
      L.nblocks = b->num_sms;
      L.smem = 0;  // set with the block shares
      nargs += L.inst.size();
      L.map_len = 3 * (size_t)L.nblocks + L.inst.size();  // bound: see plan_blocks
      nblk += L.map_len;
      plan.push_back(L);
    }
  }
  if ((rc = grow_pinned(&b->hargs, &b->args_cap, std::max<size_t>(nargs, 1)))) return rc;
  if ((rc = grow_pinned(&b->hmg, &b->mg_cap, std::max<size_t>(nargs, 1)))) return rc;
  if ((rc = grow_pinned(&b->hblk, &b->blk_cap, std::max<size_t>(nblk, 1)))) return rc;
  if (b->dargs_cap < b->args_cap) {
    if (b->dargs) CK(cudaFree(b->dargs));
    b->dargs = nullptr;
    b->dargs_cap = 0;
    CK(cudaMalloc((void**)&b->dargs, b->args_cap * sizeof(PoissonArgs)));
    b->dargs_cap = b->args_cap;
  }
  if (b->dmg_cap < b->mg_cap) {
    if (b->dmg) CK(cudaFree(b->dmg));
    b->dmg = nullptr;
    b->dmg_cap = 0;
    CK(cudaMalloc((void**)&b->dmg, b->mg_cap * sizeof(MgRebuildArgs)));
    b->dmg_cap = b->mg_cap;
  }
  if (b->dblk_cap < b->blk_cap) {
    if (b->dblk) CK(cudaFree(b->dblk));
    b->dblk = nullptr;
    b->dblk_cap = 0;
    CK(cudaMalloc((void**)&b->dblk, b->blk_cap * sizeof(int)));
    b->dblk_cap = b->blk_cap;
  }
  for (SolveLaunch& L : plan) {
    const std::vector<std::vector<int>> blocks = plan_blocks(solve_work(sims, L.inst), L.nblocks);
    if ((int)blocks.size() != L.nblocks) return fail(PB_ERR_STATE, "pb_batch_run: block plan does not cover the launch");
    std::vector<int> first(L.inst.size(), -1), count(L.inst.size(), 0);
    int* map = b->hblk + L.blk_off;
    int at = L.nblocks;
    for (int q = 0; q < L.nblocks; ++q) {
      map[q] = at;
      map[at++] = (int)blocks[q].size();
      for (int j : blocks[q]) {
        map[at++] = j;
        if (blocks[q].size() == 1) {
          if (first[j] < 0) first[j] = q;
          ++count[j];
        } else {
          first[j] = q;
          count[j] = 1;
        }
      }
    }
    L.smem = 0;
    for (size_t j = 0; j < L.inst.size(); ++j) {
      Sim* s = &sims[L.inst[j]]->s;
      const pb_step_params& p = params[(size_t)L.inst[j] * K + L.step];
      if (first[j] < 0 || count[j] > s->num_sms)
        return fail(PB_ERR_STATE, "pb_batch_run: an instance without blocks in its field-solve launch");
      PoissonArgs a = poisson_args(s, p.picard_iters, &p);
      a.blk0 = first[j];
      a.nblk = count[j];
      set_up_tiles(s, &a);
      L.smem = std::max(L.smem, mg_solve_smem_bytes(s->ncap, a.nvb, a.nblk));
      a.trace = s->trace_on ? s->ptrace : nullptr;  // traced members run without graphs
      b->hargs[L.args_off + j] = a;
      MgRebuildArgs m = mg_rebuild_args(s);
      m.blk0 = first[j];
      m.nblk = count[j];
      b->hmg[L.args_off + j] = m;
      s->batch_blocks = count[j];
    }
  }
  // ---- per-instance events
  while ((int)b->ev_inst.size() < n) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->ev_inst.push_back(e);
  }
  size_t max_launches_per_step = 1;
  {
    std::vector<int> per(K, 0);
    for (const SolveLaunch& L : plan) max_launches_per_step = std::max<size_t>(max_launches_per_step, ++per[L.step]);
  }
  while (b->ev_solve.size() < max_launches_per_step) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->ev_solve.push_back(e);
  }
  if (reports && (rc = grow_pinned(&b->hrep, &b->rep_cap, (size_t)n * K))) return rc;
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < K; ++k)
      if ((rc = check_step_params(&sims[i]->s, &params[(size_t)i * K + k]))) return rc;
  bool use_graphs = b->graphs_on != 0;
  for (int i = 0; i < n; ++i)
    if (sims[i]->s.profiling || sims[i]->s.trace_on) use_graphs = false;
  if (use_graphs) {
    // the report ring (its address is part of every graph)
    if ((size_t)K * n > b->ring_cap) {
      free_batch_graphs(b);
      if (b->ring) cudaFree(b->ring);
      if (b->hring) cudaFreeHost(b->hring);
      b->ring = nullptr; b->hring = nullptr; b->ring_cap = 0;
      const size_t cap = std::max<size_t>((size_t)K * n, 256);
      CK(cudaMalloc((void**)&b->ring, cap * sizeof(pb_step_report)));
      CK(cudaMallocHost((void**)&b->hring, cap * sizeof(pb_step_report)));
      b->ring_cap = cap;
    }
    const auto t0 = std::chrono::steady_clock::now();
    CK(cudaEventRecord(b->ev0, b->stream));
    if (nargs > 0) {
      CK(cudaMemcpyAsync(b->dargs, b->hargs, nargs * sizeof(PoissonArgs), cudaMemcpyHostToDevice, b->stream));
      CK(cudaMemcpyAsync(b->dmg, b->hmg, nargs * sizeof(MgRebuildArgs), cudaMemcpyHostToDevice, b->stream));
      CK(cudaMemcpyAsync(b->dblk, b->hblk, nblk * sizeof(int), cudaMemcpyHostToDevice, b->stream));
    }
    CK(cudaMemsetAsync(b->slot, 0, sizeof(int), b->stream));
    for (int i = 0; i < n; ++i) {
      Sim* s = &sims[i]->s;
      s->mark_used = 0;
      s->launches = 0;
      CK(cudaMemsetAsync(s->bar, 0, 2 * sizeof(unsigned int), b->stream));
      CK(cudaMemsetAsync(s->solve_ns, 0, 2 * sizeof(unsigned long long), b->stream));
    }
    b->launches = 0;
    b->last_solve_ms = -1.0;  // not timed inside graphs
    if ((rc = batch_run_graphs(b, sims, n, params, K, plan))) return rc;
    CK(cudaMemcpyAsync(b->hring, b->ring, (size_t)K * n * sizeof(pb_step_report), cudaMemcpyDeviceToHost,
                       b->stream));
    CK(cudaEventRecord(b->ev1, b->stream));
    b->last_host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    CK(cudaEventSynchronize(b->ev1));
    float gms = 0.0f;
    CK(cudaEventElapsedTime(&gms, b->ev0, b->ev1));
    b->last_ms = gms;
    for (int i = 0; i < n; ++i) {
      Sim* s = &sims[i]->s;
      b->launches += s->launches;
      if ((rc = read_counts(s))) return rc;
      if ((rc = settle_mg(s))) return rc;
      if ((rc = measure_solve(s))) return rc;
    }
    if (reports) {
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < K; ++k) reports[(size_t)i * K + k] = b->hring[(size_t)k * n + i];
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < K; ++k)
          if ((rc = check_flags(&sims[i]->s, reports[(size_t)i * K + k].errflags))) return rc;
    }
    return PB_OK;
  }
  // ---- enqueue
  while (b->tev.size() < 2 * plan.size()) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    b->tev.push_back(e);
  }
  const auto t_enq0 = std::chrono::steady_clock::now();
  CK(cudaEventRecord(b->ev0, b->stream));
  if (nargs > 0) {
    CK(cudaMemcpyAsync(b->dargs, b->hargs, nargs * sizeof(PoissonArgs), cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemcpyAsync(b->dmg, b->hmg, nargs * sizeof(MgRebuildArgs), cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemcpyAsync(b->dblk, b->hblk, nblk * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  }
  for (int i = 0; i < n; ++i) {
    Sim* s = &sims[i]->s;
    s->mark_used = 0;
    s->launches = 0;
    CK(cudaMemsetAsync(s->bar, 0, 2 * sizeof(unsigned int), b->stream));
    CK(cudaMemsetAsync(s->solve_ns, 0, 2 * sizeof(unsigned long long), b->stream));
  }
  CK(cudaEventRecord(b->ev_solve[0], b->stream));
  for (int i = 0; i < n; ++i) CK(cudaStreamWaitEvent(sims[i]->s.stream, b->ev_solve[0], 0));
  b->launches = 0;
  size_t pi = 0;
  // the members are split over the enqueue threads (member i on thread i mod T); each thread
  // keeps its first error, and the run returns the first of them
  if (!b->pool) {
    int T = b->enqueue_threads;
    if (T <= 0) T = std::max(1, std::min(8, (int)std::thread::hardware_concurrency() / 2));
    b->pool.reset(new EnqueuePool());
    b->pool->start(T - 1);
  }
  const int T = b->pool->workers() + 1;
  std::vector<int32_t> wrc(T, PB_OK);
  std::vector<std::string> werr(T);
  auto phase = [&](auto body) -> int32_t {
    std::fill(wrc.begin(), wrc.end(), PB_OK);
    b->pool->run([&](int w) {
      if (cudaSetDevice(b->device) != cudaSuccess) {
        wrc[w] = PB_ERR_CUDA;
        werr[w] = "cudaSetDevice on an enqueue thread failed";
        return;
      }
      for (int i = w; i < n && wrc[w] == PB_OK; i += T) {
        const int32_t r = body(i);
        if (r) {
          wrc[w] = r;
          werr[w] = g_err;
        }
      }
    });
    for (int w = 0; w < T; ++w)
      if (wrc[w]) {
        g_err = werr[w];
        return wrc[w];
      }
    return PB_OK;
  };
  for (int k = 0; k < K; ++k) {
    rc = phase([&](int i) -> int32_t {
      if (int32_t r = enqueue_step_pre(sims[i], &params[(size_t)i * K + k])) return r;
      CK(cudaEventRecord(b->ev_inst[i], sims[i]->s.stream));
      return PB_OK;
    });
    if (rc) return rc;
    std::vector<int> solved_by(n, -1);
    int li = 0;
    for (; pi < plan.size() && plan[pi].step == k; ++pi, ++li) {
      const SolveLaunch& L = plan[pi];
      for (int i : L.inst) {
        CK(cudaStreamWaitEvent(b->stream, b->ev_inst[i], 0));
        solved_by[i] = li;
      }
      const PoissonArgs* da = b->dargs + L.args_off;
      const int* db = b->dblk + L.blk_off;
      if ((rc = launch_mg_rebuild_batch(b, sims, L, b->dmg + L.args_off, db, false))) return rc;
      void* kargs[] = {(void*)&da, (void*)&db};
      CK(cudaEventRecord(b->tev[2 * pi], b->stream));
      if ((rc = coop_launch(b->device, b->stream, [&]() {
             return cudaLaunchCooperativeKernel((void*)k_poisson_batch, dim3(L.nblocks), dim3(PT), kargs, L.smem,
                                                b->stream);
           })))
        return rc;
      CK(cudaEventRecord(b->tev[2 * pi + 1], b->stream));
      ++b->launches;
      CK(cudaEventRecord(b->ev_solve[li], b->stream));
    }
    rc = phase([&](int i) -> int32_t {
      Sim* s = &sims[i]->s;
      if (solved_by[i] >= 0) CK(cudaStreamWaitEvent(s->stream, b->ev_solve[solved_by[i]], 0));
      if (int32_t r = enqueue_step_post(sims[i], &params[(size_t)i * K + k])) return r;
      if (reports)
        CK(cudaMemcpyAsync(&b->hrep[(size_t)i * K + k], s->rep_dev, sizeof(pb_step_report), cudaMemcpyDeviceToHost,
                           s->stream));
      return PB_OK;
    });
    if (rc) return rc;
  }
  for (int i = 0; i < n; ++i) {
    CK(cudaEventRecord(b->ev_inst[i], sims[i]->s.stream));
    CK(cudaStreamWaitEvent(b->stream, b->ev_inst[i], 0));
  }
  CK(cudaEventRecord(b->ev1, b->stream));
  b->last_host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_enq0).count();
  CK(cudaEventSynchronize(b->ev1));
  float ms = 0.0f;
  CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  b->last_ms = ms;
  b->last_solve_ms = 0.0;
  for (size_t j = 0; j < plan.size(); ++j) {
    float sm = 0.0f;
    CK(cudaEventElapsedTime(&sm, b->tev[2 * j], b->tev[2 * j + 1]));
    b->last_solve_ms += sm;
  }
  for (int i = 0; i < n; ++i) {
    Sim* s = &sims[i]->s;
    b->launches += s->launches;
    if ((rc = read_counts(s))) return rc;
    if ((rc = settle_mg(s))) return rc;
    if ((rc = measure_solve(s))) return rc;
  }
  if (reports) {
    std::memcpy(reports, b->hrep, (size_t)n * K * sizeof(pb_step_report));
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < K; ++k)
        if ((rc = check_flags(&sims[i]->s, reports[(size_t)i * K + k].errflags))) return rc;
  }
  return PB_OK;
}

int32_t pb_host_plan_blocks(const int64_t* work, int32_t m, int32_t total, int32_t* first, int32_t* count,
                            int32_t* packed) {
  if (!work || !first || !count || !packed || m < 1 || total < m)
    return fail(PB_ERR_ARG, "pb_host_plan_blocks: need work, outputs and 1 <= m <= total");
  std::vector<long> w(m);
  for (int i = 0; i < m; ++i) {
    if (work[i] < 1) return fail(PB_ERR_ARG, "pb_host_plan_blocks: costs must be positive");
    w[i] = (long)work[i];
  }
  const std::vector<std::vector<int>> blocks = plan_blocks(w, total);
  for (int i = 0; i < m; ++i) { first[i] = -1; count[i] = 0; packed[i] = 0; }
  for (int q = 0; q < (int)blocks.size(); ++q)
    for (int j : blocks[q]) {
      if (first[j] < 0) first[j] = q;
      ++count[j];
      packed[j] = blocks[q].size() > 1 ? 1 : 0;
    }
  return PB_OK;
}

int32_t pb_batch_set_threads(pb_batch* b, int32_t threads) {
  if (!b || threads < 0 || threads > 64) return fail(PB_ERR_ARG, "pb_batch_set_threads: 0 to 64 threads");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  b->pool.reset();
  b->enqueue_threads = threads;
  return PB_OK;
}

int32_t pb_batch_set_graphs(pb_batch* b, int32_t on) {
  if (!b) return fail(PB_ERR_ARG, "pb_batch_set_graphs");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  free_batch_graphs(b);
  b->graphs_on = on ? 1 : 0;
  b->graphs_broken = 0;
  b->graph_error.clear();
  return PB_OK;
}

int32_t pb_batch_graph_stats(pb_batch* b, int64_t* out3) {
  if (!b || !out3) return fail(PB_ERR_ARG, "pb_batch_graph_stats");
  out3[0] = b->graph_captures;
  out3[1] = b->graph_replays;
  out3[2] = b->graphs_broken;
  if (b->graphs_broken) g_err = b->graph_error;
  return PB_OK;
}

int32_t pb_batch_timing(pb_batch* b, double* out2) {
  if (!b || !out2) return fail(PB_ERR_ARG, "pb_batch_timing");
  out2[0] = b->last_ms;
  out2[1] = (double)b->launches;
  out2[2] = b->last_host_ms;
  out2[3] = b->last_solve_ms;
  return PB_OK;
}

int32_t pb_sim_memory(pb_sim* h, int64_t* bytes) {
  if (!h || !bytes) return fail(PB_ERR_ARG, "pb_sim_memory");
  *bytes = sim_device_bytes(&h->s);
  return PB_OK;
}

}  // extern "C"
