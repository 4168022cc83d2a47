// Batched stepping of several simulators on one GPU (included by pb_runtime.cu).
//
// The reference advances one aperture simulation per process and runs sweeps as one
// process per sweep point (Python/benchmarks/benchmark_perveance.py:78-164).  Here many
// instances share the device: each keeps its particles, fields and multigrid hierarchy
// resident and its particle kernels run on its own stream, so the kernels of different
// instances overlap.  Their field solves, which are latency-bound on one grid, run as one
// cooperative launch in which every instance gets a contiguous range of blocks with its
// own grid barrier and reductions (k_poisson_batch).

struct pb_batch {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  PoissonArgs* dargs = nullptr;  // device copy of every field-solve argument block of a run
  PoissonArgs* hargs = nullptr;  // pinned staging
  size_t args_cap = 0, dargs_cap = 0;
  int* dblk = nullptr;           // block -> argument-block maps of every launch of a run
  int* hblk = nullptr;
  size_t blk_cap = 0, dblk_cap = 0;
  pb_step_report* hrep = nullptr;  // pinned per-step reports
  size_t rep_cap = 0;
  std::vector<cudaEvent_t> ev_inst;  // per instance: "pre-solve half enqueued" / "stream done"
  std::vector<cudaEvent_t> ev_solve; // per launch of a step
  double last_ms = 0.0;
  double last_host_ms = 0.0;   // host time spent enqueuing the last run (ev0 to the last enqueue)
  long long launches = 0;
};

namespace {

struct SolveLaunch {
  int step;
  std::vector<int> inst;  // instances (indices into the run's simulator list)
  size_t args_off;        // first argument block
  size_t blk_off;         // first entry of the block map
  int nblocks;
  size_t smem;
};

// Blocks of one launch shared out in proportion to each instance's node count (at least
// one block each, at most the instance's own full-device grid).
std::vector<int> share_blocks(const std::vector<long>& work, int total) {
  const int m = (int)work.size();
  std::vector<int> nb(m, 1);
  long sum = 0;
  for (long w : work) sum += w;
  int left = total - m;
  if (left > 0 && sum > 0) {
    std::vector<std::pair<double, int>> frac;
    int given = 0;
    for (int i = 0; i < m; ++i) {
      double want = (double)left * (double)work[i] / (double)sum;
      int add = (int)want;
      nb[i] += add;
      given += add;
      frac.push_back({want - add, i});
    }
    std::sort(frac.begin(), frac.end(), [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
      return a.first > b.first || (a.first == b.first && a.second < b.second);
    });
    for (int k = 0; k < left - given && k < m; ++k) nb[frac[k].second] += 1;
  }
  // every block of the launch belongs to an instance
  int sum_nb = 0, big = 0;
  for (int i = 0; i < m; ++i) {
    sum_nb += nb[i];
    if (work[i] > work[big]) big = i;
  }
  if (m > 0 && sum_nb < total) nb[big] += total - sum_nb;
  return nb;
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
  b += (int64_t)s->nc * s->nc * 4;
  b += 4LL * (int64_t)s->sort_cap * 4 + (int64_t)s->hist_cap * 4 + 2LL * (int64_t)s->tile_cap * 8;
  b += (int64_t)s->see_cap * 16 + (int64_t)s->angle_cap * 8;
  return b;
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
  CK(cudaFuncSetAttribute((const void*)k_poisson_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)mg_coarse_smem_bytes(MG_MAX_COARSE)));
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
  if (b->dblk) cudaFree(b->dblk);
  if (b->hargs) cudaFreeHost(b->hargs);
  if (b->hblk) cudaFreeHost(b->hblk);
  if (b->hrep) cudaFreeHost(b->hrep);
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
      L.smem = 0;
      for (int i : L.inst) L.smem = std::max(L.smem, sims[i]->s.psmem);
      nargs += L.inst.size();
      nblk += (size_t)L.nblocks;
      plan.push_back(L);
    }
  }
  if ((rc = grow_pinned(&b->hargs, &b->args_cap, std::max<size_t>(nargs, 1)))) return rc;
  if ((rc = grow_pinned(&b->hblk, &b->blk_cap, std::max<size_t>(nblk, 1)))) return rc;
  if (b->dargs_cap < b->args_cap) {
    if (b->dargs) CK(cudaFree(b->dargs));
    b->dargs = nullptr;
    b->dargs_cap = 0;
    CK(cudaMalloc((void**)&b->dargs, b->args_cap * sizeof(PoissonArgs)));
    b->dargs_cap = b->args_cap;
  }
  if (b->dblk_cap < b->blk_cap) {
    if (b->dblk) CK(cudaFree(b->dblk));
    b->dblk = nullptr;
    b->dblk_cap = 0;
    CK(cudaMalloc((void**)&b->dblk, b->blk_cap * sizeof(int)));
    b->dblk_cap = b->blk_cap;
  }
  for (const SolveLaunch& L : plan) {
    std::vector<long> work;
    for (int i : L.inst) work.push_back((long)sims[i]->s.ny * sims[i]->s.nx);
    std::vector<int> nb = share_blocks(work, L.nblocks);
    int blk0 = 0;
    for (size_t j = 0; j < L.inst.size(); ++j) {
      Sim* s = &sims[L.inst[j]]->s;
      const pb_step_params& p = params[(size_t)L.inst[j] * K + L.step];
      PoissonArgs a = poisson_args(s, p.picard_iters, &p);
      if (nb[j] > s->pgrid) return fail(PB_ERR_STATE, "pb_batch_run: block share above the instance's grid");
      a.blk0 = blk0;
      a.nblk = nb[j];
      set_up_tiles(s, &a);
      a.trace = nullptr;
      b->hargs[L.args_off + j] = a;
      for (int q = 0; q < nb[j]; ++q) b->hblk[L.blk_off + blk0 + q] = (int)j;
      blk0 += nb[j];
    }
    if (blk0 != L.nblocks) return fail(PB_ERR_STATE, "pb_batch_run: block shares do not cover the launch");
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
  // ---- enqueue
  const auto t_enq0 = std::chrono::steady_clock::now();
  CK(cudaEventRecord(b->ev0, b->stream));
  if (nargs > 0) {
    CK(cudaMemcpyAsync(b->dargs, b->hargs, nargs * sizeof(PoissonArgs), cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemcpyAsync(b->dblk, b->hblk, nblk * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  }
  for (int i = 0; i < n; ++i) {
    Sim* s = &sims[i]->s;
    s->mark_used = 0;
    s->launches = 0;
    CK(cudaMemsetAsync(s->bar, 0, 2 * sizeof(unsigned int), b->stream));
  }
  CK(cudaEventRecord(b->ev_solve[0], b->stream));
  for (int i = 0; i < n; ++i) CK(cudaStreamWaitEvent(sims[i]->s.stream, b->ev_solve[0], 0));
  b->launches = 0;
  size_t pi = 0;
  for (int k = 0; k < K; ++k) {
    for (int i = 0; i < n; ++i) {
      if ((rc = enqueue_step_pre(sims[i], &params[(size_t)i * K + k]))) return rc;
      CK(cudaEventRecord(b->ev_inst[i], sims[i]->s.stream));
    }
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
      void* kargs[] = {(void*)&da, (void*)&db};
      if ((rc = coop_launch(b->device, b->stream, [&]() {
             return cudaLaunchCooperativeKernel((void*)k_poisson_batch, dim3(L.nblocks), dim3(PT), kargs, L.smem,
                                                b->stream);
           })))
        return rc;
      ++b->launches;
      CK(cudaEventRecord(b->ev_solve[li], b->stream));
    }
    for (int i = 0; i < n; ++i) {
      Sim* s = &sims[i]->s;
      if (solved_by[i] >= 0) CK(cudaStreamWaitEvent(s->stream, b->ev_solve[solved_by[i]], 0));
      if ((rc = enqueue_step_post(sims[i], &params[(size_t)i * K + k]))) return rc;
      if (reports)
        CK(cudaMemcpyAsync(&b->hrep[(size_t)i * K + k], s->rep_dev, sizeof(pb_step_report), cudaMemcpyDeviceToHost,
                           s->stream));
    }
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
  for (int i = 0; i < n; ++i) {
    Sim* s = &sims[i]->s;
    b->launches += s->launches;
    if ((rc = read_counts(s))) return rc;
  }
  if (reports) {
    std::memcpy(reports, b->hrep, (size_t)n * K * sizeof(pb_step_report));
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < K; ++k)
        if ((rc = check_flags(&sims[i]->s, reports[(size_t)i * K + k].errflags))) return rc;
  }
  return PB_OK;
}

int32_t pb_batch_timing(pb_batch* b, double* out2) {
  if (!b || !out2) return fail(PB_ERR_ARG, "pb_batch_timing");
  out2[0] = b->last_ms;
  out2[1] = (double)b->launches;
  out2[2] = b->last_host_ms;
  return PB_OK;
}

int32_t pb_sim_memory(pb_sim* h, int64_t* bytes) {
  if (!h || !bytes) return fail(PB_ERR_ARG, "pb_sim_memory");
  *bytes = sim_device_bytes(&h->s);
  return PB_OK;
}

}  // extern "C"
