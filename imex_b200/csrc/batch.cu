// Ensembles: many independent runs of uneven grid sizes advanced together.
//
// Each member is an ordinary context (its own grid, data, dt and statistics).  One step of
// the ensemble enqueues, for every member, the same sub-steps as imex_step, with two
// changes:
//   - the explicit sub-steps of the members run on a pool of streams, so small members
//     fill the GPU together;
//   - each implicit solve of a stage (the magnetic system, the one or two pressure solves)
//     is ONE cooperative launch for all members, in which every member owns a contiguous
//     range of CTAs with its own barrier and reductions (see batch_solve_build).  Members
//     never wait on one another, and no two cooperative kernels run at the same time.
// The explicit sub-steps run in one of two ways:
//   - batched (streams = 0, the default): each explicit sub-step is ONE launch for all
//     members.  The step is planned once: every member's launch functions run in recording
//     mode (launch.cuh), and the launches the members recorded for a sub-step become one
//     launch of the same kernel body over all their grids, laid end to end;
//   - on a pool of streams (streams > 0): every member launches its own kernels, members
//     spread over the streams.
// The whole step is captured once into a CUDA graph and replayed; if capture fails the
// same step is launched directly and the reason is kept (imex_batch_last_error).
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "imex_internal.h"
#include "launch.cuh"

struct imex_batch {
  std::vector<imex_ctx*> members;
  std::vector<cudaStream_t> streams;  // streams of the explicit sub-steps
  cudaStream_t origin = nullptr;      // joins the members around the batched solves
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
  imex::BatchSolvePlan* mag = nullptr;
  imex::BatchSolvePlan* pres = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // the planned step of the batched mode: its launches in order, and their device tables
  std::vector<imex::PlanItem> plan;
  imex::PlanArena arena;
  int nstreams = 0;  // 0: batched explicit sub-steps; > 0: streams of the per-member launches
  int solve_tile = 0;  // tile shape of the batched B-form solve (kBatchTileX / kBatchTileY)
  bool use_graph = true;
  bool members_on_batch = false;  // the members' streams are the batch's (pool or origin)
  bool prepared = false;
  bool graph_ok = false;
  std::string last_error;
};

namespace imex {

__global__ void k_copies(const CopyDesc* __restrict__ d) {
  const CopyDesc c = d[blockIdx.y];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < c.n; i += (long long)gridDim.x * blockDim.x)
    c.dst[i] = c.src[i];
}

imex_status plan_alloc(PlanArena& arena, size_t bytes, void** p, std::string& err) {
  *p = nullptr;
  cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    err = std::string("batched launch tables: ") + cudaGetErrorString(e);
    return IMEX_ERR_CUDA;
  }
  arena.dev.push_back(*p);
  return IMEX_OK;
}
imex_status plan_upload(void* dst, const void* src, size_t bytes, std::string& err) {
  cudaError_t e = bytes ? cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) : cudaSuccess;
  if (e != cudaSuccess) {
    err = std::string("batched launch tables: ") + cudaGetErrorString(e);
    return IMEX_ERR_CUDA;
  }
  return IMEX_OK;
}
cudaError_t copy_d2d(imex_ctx* ctx, double* dst, const double* src, long long n) {
  if (ctx->rec) {
    RecOp op;
    op.copy = CopyDesc{dst, src, n};
    ctx->rec->ops.push_back(std::move(op));
    return cudaSuccess;
  }
  return cudaMemcpyAsync(dst, src, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
}

}  // namespace imex

namespace {

using namespace imex;

constexpr unsigned kCopyThreads = 256;
cudaError_t launch_copies(const PlanItem& it, cudaStream_t s) {
  k_copies<<<dim3(it.nblocks, it.gy), it.block, 0, s>>>(static_cast<const CopyDesc*>(it.args));
  return cudaGetLastError();
}

imex_status berr(imex_batch* b, imex_status s, const std::string& msg) {
  if (b) b->last_error = msg;
  return s;
}
imex_status bcheck(imex_batch* b, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return IMEX_OK;
  return berr(b, IMEX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
// a member's failure, with its message
imex_status merr(imex_batch* b, size_t m, imex_status s) {
  if (s != IMEX_OK) b->last_error = "member " + std::to_string(m) + ": " + b->members[m]->last_error;
  return s;
}

// Drop the streams, plans and graph.  Members that are still alive first get a stream of
// their own again: they must never hold a handle to a destroyed batch stream.
void release_plans(imex_batch* b, bool members_alive) {
  if (members_alive && b->members_on_batch)
    for (imex_ctx* c : b->members) imex_set_stream(c, nullptr);
  b->members_on_batch = false;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  batch_solve_free(b->mag);
  batch_solve_free(b->pres);
  for (void* p : b->arena.dev) cudaFree(p);
  b->arena.dev.clear();
  b->plan.clear();
  b->mag = b->pres = nullptr;
  for (cudaStream_t s : b->streams) cudaStreamDestroy(s);
  for (cudaEvent_t e : b->ev_join) cudaEventDestroy(e);
  b->streams.clear();
  b->ev_join.clear();
  b->prepared = false;
  b->graph_ok = false;
}

// The sub-steps of one ensemble step (main.cpp:335-561 per member), in order: `group`
// runs a per-member launch function for every member, `solve` one batched solve
// (BATCH_MAGNETIC / BATCH_PRESSURE) for all of them.
template <class G, class V>
imex_status step_sequence(imex_batch* b, G group, V solve) {
  const DevParams& P = b->members[0]->P;
  imex_status s;
  if ((s = group([](imex_ctx* c) { return launch_step_prologue(c); })) != IMEX_OK) return s;
  for (int r = 0; r < P.RKs; ++r) {
    s = group([r](imex_ctx* c) {
      imex_status t = launch_stage_combine(c, r);
      if (t == IMEX_OK) t = launch_reconstruct(c, false);
      if (t == IMEX_OK) t = launch_flux_update(c, 0);
      if (t == IMEX_OK) t = mag_rhs(c);
      return t;
    });
    if (s != IMEX_OK || (s = solve(BATCH_MAGNETIC)) != IMEX_OK) return s;
    s = group([](imex_ctx* c) {
      imex_status t = mag_out(c);
      if (t == IMEX_OK && c->P.Energy_Modify)
        t = cuda_check(c, copy_d2d(c, c->Bsave, c->cons + 5 * c->N, 3 * (long long)c->N), "Bsave");
      if (t == IMEX_OK) t = launch_flux_update(c, second_flux_form(c));
      if (t == IMEX_OK) t = pres_part1(c);
      return t;
    });
    if (s != IMEX_OK || (s = solve(BATCH_PRESSURE)) != IMEX_OK) return s;
    bool second = false;
    s = group([r, &second](imex_ctx* c) { return pres_part2(c, r, &second); });
    if (s != IMEX_OK) return s;
    if (second && (s = solve(BATCH_PRESSURE)) != IMEX_OK) return s;
    s = group([r](imex_ctx* c) {
      imex_status t = pres_part3(c);
      if (t == IMEX_OK && c->P.magfield == IMEX_StaggerCT) t = launch_ct(c, 0);
      else if (t == IMEX_OK && c->P.magfield == IMEX_UnStaggerCT) t = launch_ct(c, 1);
      if (t == IMEX_OK) t = launch_stage_derivative(c, r);
      return t;
    });
    if (s != IMEX_OK) return s;
  }
  return IMEX_OK;
}
BatchSolvePlan* solve_plan(imex_batch* b, int kind) { return kind == BATCH_MAGNETIC ? b->mag : b->pres; }

// one step of every member on the pool of streams, enqueued without a host wait
imex_status enqueue_step_streams(imex_batch* b) {
  cudaError_t e = cudaSuccess;
  auto fork = [&]() {
    e = cudaEventRecord(b->ev_fork, b->origin);
    for (cudaStream_t s : b->streams)
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s, b->ev_fork, 0);
    return bcheck(b, e, "batch fork");
  };
  auto join = [&]() {
    for (size_t k = 0; k < b->streams.size(); ++k) {
      if (e == cudaSuccess) e = cudaEventRecord(b->ev_join[k], b->streams[k]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(b->origin, b->ev_join[k], 0);
    }
    return bcheck(b, e, "batch join");
  };
  auto group = [&](auto f) {
    for (size_t m = 0; m < b->members.size(); ++m) {
      imex_status s = f(b->members[m]);
      if (s != IMEX_OK) return merr(b, m, s);
    }
    return IMEX_OK;
  };
  imex_ctx* c0 = b->members[0];
  auto solve = [&](int kind) {
    imex_status s;
    if ((s = join()) != IMEX_OK) return s;
    if ((s = batch_solve_run(solve_plan(b, kind), b->origin, c0)) != IMEX_OK)
      return berr(b, s, b->last_error.empty() ? c0->last_error : b->last_error);
    return fork();
  };
  imex_status s = fork();
  if (s == IMEX_OK) s = step_sequence(b, group, solve);
  if (s != IMEX_OK) return s;
  return join();
}

// The launches that the members recorded for one group of sub-steps, as launches of the
// planned step.  Round k takes the k-th recorded operation of every member; operations of
// a round that run the same kernel body (or are copies) become one launch.  A member's
// operations therefore run in its own order, one round after another.
imex_status flush_records(imex_batch* b, const std::vector<Recorder>& R) {
  std::vector<size_t> idx(R.size(), 0);
  std::string err;
  for (;;) {
    std::vector<std::pair<const void*, std::vector<const RecOp*>>> groups;
    for (size_t m = 0; m < R.size(); ++m) {
      if (idx[m] >= R[m].ops.size()) continue;
      const RecOp* op = &R[m].ops[idx[m]++];
      const void* key = op->plan ? reinterpret_cast<const void*>(op->plan) : nullptr;
      auto g = groups.begin();
      while (g != groups.end() && g->first != key) ++g;
      if (g == groups.end()) groups.push_back({key, {op}});
      else g->second.push_back(op);
    }
    if (groups.empty()) return IMEX_OK;
    for (auto& g : groups) {
      PlanItem it;
      imex_status s = IMEX_OK;
      if (g.first) {
        s = g.second[0]->plan(g.second, b->arena, it, err);
      } else {
        std::vector<CopyDesc> d;
        long long nmax = 1;
        for (const RecOp* op : g.second) {
          d.push_back(op->copy);
          if (op->copy.n > nmax) nmax = op->copy.n;
        }
        void* dd = nullptr;
        s = plan_alloc(b->arena, d.size() * sizeof(CopyDesc), &dd, err);
        if (s == IMEX_OK) s = plan_upload(dd, d.data(), d.size() * sizeof(CopyDesc), err);
        long long nb = (nmax + 4 * kCopyThreads - 1) / (4 * kCopyThreads);
        it.launch = &launch_copies;
        it.args = dd;
        it.nblocks = (unsigned)(nb < 1024 ? nb : 1024);
        it.gy = (unsigned)d.size();
        it.block = kCopyThreads;
      }
      if (s != IMEX_OK) return berr(b, s, err);
      b->plan.push_back(it);
    }
  }
}

// Plan one step of the batched mode: record every member's launches group by group and
// turn them into batched launches (device tables are built here, outside any capture).
imex_status plan_step(imex_batch* b) {
  b->plan.clear();
  auto group = [&](auto f) {
    std::vector<Recorder> R(b->members.size());
    for (size_t m = 0; m < b->members.size(); ++m) {
      imex_ctx* c = b->members[m];
      c->rec = &R[m];
      imex_status s = f(c);
      c->rec = nullptr;
      if (s != IMEX_OK) return merr(b, m, s);
    }
    return flush_records(b, R);
  };
  auto solve = [&](int kind) {
    PlanItem it;
    it.solve = kind;
    b->plan.push_back(it);
    return IMEX_OK;
  };
  return step_sequence(b, group, solve);
}
imex_status enqueue_step_planned(imex_batch* b) {
  imex_ctx* c0 = b->members[0];
  for (const PlanItem& it : b->plan) {
    if (it.solve >= 0) {
      imex_status s = batch_solve_run(solve_plan(b, it.solve), b->origin, c0);
      if (s != IMEX_OK) return berr(b, s, b->last_error.empty() ? c0->last_error : b->last_error);
      continue;
    }
    cudaError_t e = it.launch(it, b->origin);
    if (e != cudaSuccess) return bcheck(b, e, "batched launch");
  }
  return IMEX_OK;
}
imex_status enqueue_step(imex_batch* b) {
  return b->nstreams == 0 ? enqueue_step_planned(b) : enqueue_step_streams(b);
}

// streams, batched-solve plans and (if asked) the captured step
imex_status prepare(imex_batch* b) {
  if (b->prepared) return IMEX_OK;
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < b->nstreams && e == cudaSuccess; ++k) {
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (s) b->streams.push_back(s);
    if (ev) b->ev_join.push_back(ev);
  }
  if (e != cudaSuccess) return bcheck(b, e, "batch streams");
  // members run on the pool (streams mode) or on the batch's own stream (batched mode)
  for (size_t m = 0; m < b->members.size(); ++m) {
    cudaStream_t st = b->streams.empty() ? b->origin : b->streams[m % b->streams.size()];
    imex_status s = imex_set_stream(b->members[m], st);
    if (s != IMEX_OK) return merr(b, m, s);
    b->members[m]->prof_on = false;
  }
  b->members_on_batch = true;
  imex_status s = batch_solve_build(b->members, BATCH_MAGNETIC, &b->mag, b->solve_tile);
  if (s == IMEX_OK) s = batch_solve_build(b->members, BATCH_PRESSURE, &b->pres);
  if (s != IMEX_OK) return berr(b, s, "batched solve set-up: " + b->members[0]->last_error);
  if (b->nstreams == 0 && (s = plan_step(b)) != IMEX_OK) return s;
  b->prepared = true;
  b->graph_ok = false;
  if (!b->use_graph) return IMEX_OK;
  // capture one step; on failure keep the reason and launch directly instead
  e = cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    b->last_error = std::string("graph capture unavailable: ") + cudaGetErrorString(e);
    cudaGetLastError();
    return IMEX_OK;
  }
  imex_status cs = enqueue_step(b);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(b->origin, &g);
  if (cs == IMEX_OK && e == cudaSuccess && g) e = cudaGraphInstantiate(&b->exec, g, 0);
  if (cs != IMEX_OK || e != cudaSuccess || !g) {
    // no graph: start again from fresh streams (a failed capture can leave them unusable)
    const std::string why = cs != IMEX_OK ? b->last_error : std::string(cudaGetErrorString(e));
    if (g) cudaGraphDestroy(g);
    b->exec = nullptr;
    cudaGetLastError();
    release_plans(b, true);
    b->use_graph = false;
    imex_status r = prepare(b);
    b->last_error = "graph capture failed, launching directly: " + why;
    return r;
  }
  b->graph = g;
  b->graph_ok = true;
  return IMEX_OK;
}

// worst status of the members since the last check (synchronises)
imex_status members_status(imex_batch* b) {
  cudaError_t e = cudaStreamSynchronize(b->origin);
  if (e != cudaSuccess) return bcheck(b, e, "batch step");
  imex_status worst = IMEX_OK;
  for (size_t m = 0; m < b->members.size(); ++m) {
    imex_solve_stats st;
    imex_status s = imex_get_stats(b->members[m], &st);
    if (s != IMEX_OK) return merr(b, m, s);
    if (st.status != IMEX_OK && worst == IMEX_OK) {
      worst = (imex_status)st.status;
      b->last_error = "member " + std::to_string(m) + ": " + imex_status_string(worst);
    }
  }
  if (worst != IMEX_OK)
    for (imex_ctx* c : b->members) imex_reset_stats(c);
  return worst;
}

// device copies of every member's step state, to run trial steps and come back
struct Snapshot {
  std::vector<double*> planes;
  std::vector<std::vector<unsigned char>> scalars;
};
imex_status take_snapshot(imex_batch* b, Snapshot& snap, bool restore) {
  for (size_t m = 0; m < b->members.size(); ++m) {
    imex_ctx* c = b->members[m];
    const size_t N = c->N;
    if (!restore) {
      double* p = nullptr;
      cudaError_t e = cudaMalloc(&p, 13 * N * sizeof(double));
      if (e != cudaSuccess) return bcheck(b, e, "autotune snapshot");
      snap.planes.push_back(p);
      snap.scalars.emplace_back(sizeof(DevScalars));
    }
    double* p = snap.planes[m];
    auto cp = [&](double* dst, const double* src, size_t n) {
      return cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, b->origin);
    };
    cudaError_t e;
    if (!restore) {
      e = cp(p, c->prim, 8 * N);
      if (e == cudaSuccess) e = cp(p + 8 * N, c->bx, N);
      if (e == cudaSuccess) e = cp(p + 9 * N, c->by, N);
      if (e == cudaSuccess) e = cp(p + 10 * N, c->A, 3 * N);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(snap.scalars[m].data(), c->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, b->origin);
    } else {
      e = cp(c->prim, p, 8 * N);
      if (e == cudaSuccess) e = cp(c->bx, p + 8 * N, N);
      if (e == cudaSuccess) e = cp(c->by, p + 9 * N, N);
      if (e == cudaSuccess) e = cp(c->A, p + 10 * N, 3 * N);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->sc, snap.scalars[m].data(), sizeof(DevScalars), cudaMemcpyHostToDevice, b->origin);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->origin);
    if (e != cudaSuccess) return bcheck(b, e, "autotune snapshot copy");
  }
  return IMEX_OK;
}

}  // namespace

extern "C" {

imex_status imex_batch_create(const imex_config* cfg, int members, const int* nx, const int* ny,
                              imex_batch** out) {
  if (!cfg || members < 1 || !nx || !ny || !out) return IMEX_ERR_INVALID;
  *out = nullptr;
  imex_batch* b = new (std::nothrow) imex_batch();
  if (!b) return IMEX_ERR_CUDA;
  cudaError_t e = cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    imex_batch_destroy(b);
    return IMEX_ERR_CUDA;
  }
  for (int m = 0; m < members; ++m) {
    imex_ctx* c = nullptr;
    imex_status s = imex_create(cfg, nx[m], ny[m], &c);
    if (s != IMEX_OK) {
      imex_batch_destroy(b);
      return s;
    }
    b->members.push_back(c);
  }
  *out = b;
  return IMEX_OK;
}

imex_status imex_batch_destroy(imex_batch* b) {
  if (!b) return IMEX_ERR_INVALID;
  if (b->origin) cudaStreamSynchronize(b->origin);
  for (imex_ctx* c : b->members) imex_destroy(c);
  b->members.clear();
  release_plans(b, false);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->origin) cudaStreamDestroy(b->origin);
  delete b;
  return IMEX_OK;
}

imex_status imex_batch_member(imex_batch* b, int m, imex_ctx** ctx) {
  if (!b || !ctx || m < 0 || m >= (int)b->members.size()) return IMEX_ERR_INVALID;
  *ctx = b->members[m];
  return IMEX_OK;
}

const char* imex_batch_last_error(const imex_batch* b) { return b ? b->last_error.c_str() : "no batch"; }

imex_status imex_batch_configure(imex_batch* b, int streams, int use_graph) {
  if (!b || streams < 0 || streams > 64) return IMEX_ERR_INVALID;
  if (b->origin) cudaStreamSynchronize(b->origin);
  release_plans(b, true);
  b->nstreams = streams;
  b->use_graph = use_graph != 0;
  return IMEX_OK;
}

imex_status imex_batch_step(imex_batch* b, int steps, double* device_ms) {
  if (!b || steps < 0) return IMEX_ERR_INVALID;
  for (imex_ctx* c : b->members)
    if (c->P.RKs != b->members[0]->P.RKs || c->P.magfield != b->members[0]->P.magfield)
      return berr(b, IMEX_ERR_INVALID, "members differ in RK stages or magnetic form");
  imex_status s = prepare(b);
  if (s != IMEX_OK) return s;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  cudaError_t e = cudaEventCreate(&t0);
  if (e == cudaSuccess) e = cudaEventCreate(&t1);
  if (e == cudaSuccess) e = cudaEventRecord(t0, b->origin);
  for (int k = 0; k < steps && e == cudaSuccess && s == IMEX_OK; ++k) {
    if (b->graph_ok) e = cudaGraphLaunch(b->exec, b->origin);
    else s = enqueue_step(b);
  }
  if (e == cudaSuccess) e = cudaEventRecord(t1, b->origin);
  if (e == cudaSuccess) e = cudaEventSynchronize(t1);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  if (s != IMEX_OK) return s;
  if (e != cudaSuccess) return bcheck(b, e, "batch step");
  if (device_ms) *device_ms = ms;
  return members_status(b);
}

imex_status imex_batch_info(imex_batch* b, int* streams, int* graph_used, int* solve_launches_per_step) {
  if (!b) return IMEX_ERR_INVALID;
  if (streams) *streams = b->nstreams;
  if (graph_used) *graph_used = b->graph_ok ? 1 : 0;
  if (solve_launches_per_step) {
    int n = 0;
    if (b->mag) n += (int)b->mag->chunks.size();
    if (b->pres) n += (int)b->pres->chunks.size();
    *solve_launches_per_step = n;
  }
  return IMEX_OK;
}

imex_status imex_batch_explicit_launches(imex_batch* b, int* launches_per_step, int* solve_launches_per_step) {
  if (!b || !launches_per_step) return IMEX_ERR_INVALID;
  imex_status s = prepare(b);
  if (s != IMEX_OK) return s;
  int n = -1;
  if (b->nstreams == 0) {
    n = 0;
    for (const PlanItem& it : b->plan) n += it.solve < 0 ? 1 : 0;
  }
  *launches_per_step = n;
  if (solve_launches_per_step) {  // a chunk of a batched solve: a barrier reset and the solve
    int m = 0;
    for (const PlanItem& it : b->plan)
      if (it.solve >= 0) m += 2 * (int)solve_plan(b, it.solve)->chunks.size();
    *solve_launches_per_step = b->nstreams == 0 ? m : -1;
  }
  return IMEX_OK;
}

imex_status imex_batch_set_solve_tile(imex_batch* b, int tile) {
  if (!b || tile < 0 || tile >= kBatchTiles) return IMEX_ERR_INVALID;
  if (b->origin) cudaStreamSynchronize(b->origin);
  release_plans(b, true);
  b->solve_tile = tile;
  return IMEX_OK;
}

imex_status imex_batch_autotune(imex_batch* b, int trial_steps, imex_batch_tuning* out) {
  if (!b || trial_steps < 1) return IMEX_ERR_INVALID;
  imex_ctx* c0 = b->members[0];
  const int restart0 = c0->cfg.gmres_restart;
  // in mixed precision, whether the magnetic systems take the FP32 form pays only where
  // FP64 GMRES needs many Krylov steps: time both
  const int solves0 = c0->cfg.mixed_solves;
  const int mag = IMEX_MIXED_MAGNETIC | IMEX_MIXED_MAGNETIC_B;
  // the tile shape matters for the B-form solve of the fast arithmetic, the one with choices
  const bool tiles = c0->P.magfield != IMEX_PotentialA && c0->P.fast;
  struct Choice {
    int streams, restart, solves, tile;
  };
  Choice best{b->nstreams, restart0, solves0, b->solve_tile};
  double best_ms = 1e300;
  Snapshot snap;
  imex_status s = take_snapshot(b, snap, false);
  auto trial = [&](const Choice& c) {
    for (imex_ctx* m : b->members) {
      m->cfg.gmres_restart = c.restart;
      m->cfg.mixed_solves = c.solves;
    }
    b->solve_tile = c.tile;
    if (s == IMEX_OK) s = imex_batch_configure(b, c.streams, b->use_graph ? 1 : 0);
    double ms = 0.0;
    if (s == IMEX_OK) s = imex_batch_step(b, 1, nullptr);  // warm-up (and graph capture)
    if (s == IMEX_OK) s = imex_batch_step(b, trial_steps, &ms);
    if (s == IMEX_OK) s = take_snapshot(b, snap, true);
    if (s == IMEX_OK && ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  };
  // one choice at a time, each from the best so far: explicit mode, solve tile, restart
  // length, FP32 magnetic solves
  for (int sc : {0, 4, 8, 16}) trial(Choice{sc, restart0, solves0, 0});
  if (tiles)
    for (int t = 1; t < kBatchTiles; ++t) trial(Choice{best.streams, best.restart, best.solves, t});
  if (restart0 > 15) trial(Choice{best.streams, 15, best.solves, best.tile});
  if (c0->cfg.precision == IMEX_PRECISION_MIXED)
    trial(Choice{best.streams, best.restart, (best.solves & mag) ? (best.solves & ~mag) : (best.solves | IMEX_MIXED_MAGNETIC_B),
                 best.tile});
  for (double* p : snap.planes) cudaFree(p);
  for (imex_ctx* m : b->members) {
    m->cfg.gmres_restart = best.restart;
    m->cfg.mixed_solves = best.solves;
  }
  b->solve_tile = best.tile;
  imex_status s2 = imex_batch_configure(b, best.streams, b->use_graph ? 1 : 0);
  if (s != IMEX_OK) return s;
  if (s2 != IMEX_OK) return s2;
  if (out) {
    out->streams = best.streams;
    out->gmres_restart = best.restart;
    out->ms_per_step = best_ms / trial_steps;
    out->mixed_solves = best.solves;
    out->solve_tile_x = kBatchTileX[best.tile];
    out->solve_tile_y = kBatchTileY[best.tile];
  }
  return IMEX_OK;
}

}  // extern "C"
