// Batched multiplication: many independent C_b = A_b . B_b (FP64) in one
// persistent launch over a global work queue, replayed from a captured CUDA
// graph, with the launch shape picked by an autotuner.  No reference
// counterpart (the reference multiplies one matrix pair per call).
//
// Creation runs the symbolic phase of every instance (C patterns, stacks,
// work lists) with the current values.  lamb_gpu_batch_execute replays the
// numeric phase only (product-filter decisions and C patterns frozen at
// creation); lamb_gpu_batch_run with LAMB_GPU_BATCH_FULL redoes the whole
// multiply of every instance -- symbolic phase from the current values, the
// graph-replayed numeric launch, result filter -- and times the three parts.
// The graph reads the work queue and the instance table from device arrays,
// so a full run refreshes their contents in place; the graph is captured
// again only when the queue's length changes.  The autotuner picks the
// launch shape (warps per CTA, stack entries per column-table chunk, items
// per queue fetch) and the queue order: instance-major (largest instance
// first) or grouped by C block shape (M, N).
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <numeric>
#include <sstream>
#include <string>

#include "multiply.cuh"

namespace lamb {

struct Batch {
  Ctx* ctx = nullptr;
  double eps = 0.0;
  std::vector<DevMatrix*> a, b, c;
  std::vector<double*> nrm;          // C block norms of every instance
  std::vector<int64_t> nrm_cap;
  std::vector<int> order;            // instance order of the instance-major queue
  bool by_shape = false;             // queue grouped by C block shape (autotuned)
  // Every operand's handle and layout generation at creation: the graph holds
  // their raw device pointers, so an execution is refused once any of them
  // was destroyed, re-laid-out or reallocated.
  std::vector<lamb_gpu_matrix> handles;
  std::vector<uint64_t> gens;
  std::vector<Symbolic> sym;
  Work* work = nullptr;
  int32_t* work_c = nullptr;
  int32_t* work_i = nullptr;
  BatchInst* inst = nullptr;
  unsigned long long* head = nullptr;
  int64_t n_work = 0, n_products = 0;
  double flops = 0;
  int max_inner = 1;
  BatchConfig cfg;
  bool tuned = false;
  float tuned_ms = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

// ---- autotune cache (process-wide, optionally persisted) --------------------------
static std::mutex g_tune_mu;
static std::map<std::string, BatchConfig> g_tune;

static std::string tune_signature(const Batch& b) {
  // bucket the queue length to powers of two; the inner-size class matters
  int64_t q = 1;
  while (q < b.n_work) q <<= 1;
  std::ostringstream os;
  os << "q" << q << "_k" << b.max_inner << "_n" << b.c.size();
  return os.str();
}

static void load_tune_file() {
  const char* path = getenv("LAMB_GPU_AUTOTUNE_CACHE");
  if (!path) return;
  FILE* f = fopen(path, "r");
  if (!f) return;
  char key[256];
  int w, c, g;
  while (fscanf(f, "%255s %d %d %d", key, &w, &c, &g) == 4) g_tune[key] = BatchConfig{w, c, g};
  fclose(f);
}

static void store_tune_file(const std::string& key, const BatchConfig& cfg) {
  const char* path = getenv("LAMB_GPU_AUTOTUNE_CACHE");
  if (!path) return;
  FILE* f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "%s %d %d %d\n", key.c_str(), cfg.warps, cfg.cap, cfg.grab);
  fclose(f);
}

// Queue grouped by C block shape: items stably sorted by (M, N) (bits 40..55
// of Work::lo), in place.
__global__ void k_shape_keys(int64_t n, const Work* __restrict__ w, uint16_t* __restrict__ key,
                             int64_t* __restrict__ idx) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    key[i] = (uint16_t)((unsigned long long)w[i].lo >> 40);
    idx[i] = i;
  }
}
__global__ void k_gather_queue(int64_t n, const int64_t* __restrict__ idx, const Work* __restrict__ w,
                               const int32_t* __restrict__ wc, const int32_t* __restrict__ wi, Work* __restrict__ w2,
                               int32_t* __restrict__ wc2, int32_t* __restrict__ wi2) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = idx[i];
    w2[i] = w[j];
    wc2[i] = wc[j];
    wi2[i] = wi[j];
  }
}

static int32_t sort_by_shape(Batch* B) {
  Ctx* ctx = B->ctx;
  const int64_t n = B->n_work;
  if (n <= 1) return LAMB_GPU_OK;
  uint16_t *k0 = nullptr, *k1 = nullptr;
  int64_t *i0 = nullptr, *i1 = nullptr;
  Work* w2 = nullptr;
  int32_t *wc2 = nullptr, *wi2 = nullptr;
  void* tmp = nullptr;
  struct F {
    Ctx* ctx;
    std::vector<void**> p;
    ~F() { for (auto q : p) { if (*q) cudaFreeAsync(*q, ctx->stream); *q = nullptr; } }
  } fr{ctx, {(void**)&k0, (void**)&k1, (void**)&i0, (void**)&i1, (void**)&w2, (void**)&wc2, (void**)&wi2, &tmp}};
  LAMB_TRY(dalloc(ctx, &k0, n)); LAMB_TRY(dalloc(ctx, &k1, n));
  LAMB_TRY(dalloc(ctx, &i0, n)); LAMB_TRY(dalloc(ctx, &i1, n));
  LAMB_TRY(dalloc(ctx, &w2, n)); LAMB_TRY(dalloc(ctx, &wc2, n)); LAMB_TRY(dalloc(ctx, &wi2, n));
  k_shape_keys<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, B->work, k0, i0);
  LAMB_LAUNCHED(ctx);
  size_t bytes = 0;
  LAMB_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, bytes, k0, k1, i0, i1, n, 0, 16, ctx->stream));
  LAMB_TRY(dalloc(ctx, (char**)&tmp, (int64_t)bytes + 16));
  LAMB_CUDA(ctx, cub::DeviceRadixSort::SortPairs(tmp, bytes, k0, k1, i0, i1, n, 0, 16, ctx->stream));
  k_gather_queue<<<grid_for(n), kThreads, 0, ctx->stream>>>(n, i1, B->work, B->work_c, B->work_i, w2, wc2, wi2);
  LAMB_LAUNCHED(ctx);
  LAMB_CUDA(ctx, cudaMemcpyAsync(B->work, w2, sizeof(Work) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  LAMB_CUDA(ctx, cudaMemcpyAsync(B->work_c, wc2, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  LAMB_CUDA(ctx, cudaMemcpyAsync(B->work_i, wi2, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  return LAMB_GPU_OK;
}

static int32_t run_once(Batch* B, const BatchConfig& cfg, int64_t n_items) {
  Ctx* ctx = B->ctx;
  LAMB_CUDA(ctx, cudaMemsetAsync(B->head, 0, sizeof(unsigned long long), ctx->stream));
  return launch_batch(ctx, n_items, B->work, B->work_c, B->work_i, B->inst, B->head, cfg, B->max_inner);
}

// Times every candidate shape on a prefix of the queue (at most an eighth of
// it, at least all of a small queue; one warm-up and one timed launch each)
// and keeps the fastest.
static int32_t autotune(Batch* B) {
  Ctx* ctx = B->ctx;
  const std::string key = tune_signature(*B);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    static bool loaded = false;
    if (!loaded) { load_tune_file(); loaded = true; }
    auto it = g_tune.find(key);
    if (it != g_tune.end()) { B->cfg = it->second; B->tuned = true; return LAMB_GPU_OK; }
  }
  float best = 1e30f;
  BatchConfig best_cfg;
  const int64_t sample = B->n_work < (1 << 20) ? B->n_work : std::max<int64_t>(1 << 20, B->n_work / 8);
  for (int w : {4, 8})
    for (int cap : {16, 32})
      for (int grab : {1, 4, 16}) {
        BatchConfig cfg{w, cap, grab};
        LAMB_TRY(run_once(B, cfg, sample));
        LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[5], ctx->stream));
        LAMB_TRY(run_once(B, cfg, sample));
        LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[6], ctx->stream));
        LAMB_CUDA(ctx, cudaEventSynchronize(ctx->ev[6]));
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[5], ctx->ev[6]);
        if (ms < best) { best = ms; best_cfg = cfg; }
      }
  B->cfg = best_cfg;
  B->tuned = true;
  B->tuned_ms = best;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune[key] = best_cfg;
  store_tune_file(key, best_cfg);
  return LAMB_GPU_OK;
}

static void destroy_batch(Batch* B) {
  if (!B) return;
  Ctx* ctx = B->ctx;
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  for (auto& s : B->sym) free_symbolic(ctx, s);
  for (auto& p : B->nrm) dfree(ctx, p);
  dfree(ctx, B->work);
  dfree(ctx, B->work_c);
  dfree(ctx, B->work_i);
  dfree(ctx, B->inst);
  dfree(ctx, B->head);
  cudaStreamSynchronize(ctx->stream);
  delete B;
}

__global__ void k_fill_i32(int64_t n, int32_t v, int32_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = v;
}

// Symbolic phase of every instance from the current values, its work list,
// the global queue (instance-major, largest instance first; grouped by C
// block shape when B->by_shape) and the instance table.  *relayout tells
// whether the queue's length changed (the graph must then be captured again).
static int32_t build_queue(Batch* B, bool first, bool* relayout) {
  Ctx* ctx = B->ctx;
  const int n = (int)B->c.size();
  std::vector<Work*> works(n, nullptr);
  std::vector<int32_t*> wcs(n, nullptr);
  std::vector<BatchInst> hinst(n);
  struct Free {
    Ctx* ctx;
    std::vector<Work*>* w;
    std::vector<int32_t*>* c;
    ~Free() {
      for (auto& p : *w) dfree(ctx, p);
      for (auto& p : *c) dfree(ctx, p);
    }
  } fr{ctx, &works, &wcs};
  const bool filt = B->eps > 0;
  int64_t n_work = 0, n_products = 0;
  double flops = 0.0;
  for (int i = 0; i < n; ++i) {
    free_symbolic(ctx, B->sym[i]);
    B->sym[i] = Symbolic{};
    int64_t* a_offk = nullptr;
    LAMB_TRY(pack_offk(ctx, B->a[i], true, &a_offk));
    int32_t rc = symbolic_phase(ctx, B->a[i], B->b[i], B->c[i], B->eps, filt, false, a_offk, &B->sym[i]);
    dfree(ctx, a_offk);
    LAMB_TRY(rc);
    LAMB_TRY(build_work(ctx, B->c[i], B->sym[i], B->a[i], &works[i], &wcs[i]));
    const int64_t m = B->sym[i].c_nnz;
    if (B->nrm_cap[i] < m) {
      dfree(ctx, B->nrm[i]);
      LAMB_TRY(dalloc(ctx, &B->nrm[i], std::max<int64_t>(m, 1)));
      B->nrm_cap[i] = std::max<int64_t>(m, 1);
    }
    n_work += m;
    n_products += B->sym[i].n_ent;
    flops += B->sym[i].flops;
    B->max_inner = std::max(B->max_inner, max_block(B->a[i]->h_col_bs));
    hinst[i] = BatchInst{B->sym[i].ent, B->a[i]->data, B->b[i]->data, B->c[i]->data, B->nrm[i]};
    B->c[i]->norms_valid = false;
  }
  if (first) {
    B->order.resize(n);
    std::iota(B->order.begin(), B->order.end(), 0);
    std::stable_sort(B->order.begin(), B->order.end(),
                     [&](int x, int y) { return B->sym[x].flops > B->sym[y].flops; });
  }
  *relayout = n_work != B->n_work || !B->work;
  if (*relayout) {
    dfree(ctx, B->work);
    dfree(ctx, B->work_c);
    dfree(ctx, B->work_i);
    LAMB_TRY(dalloc(ctx, &B->work, std::max<int64_t>(n_work, 1)));
    LAMB_TRY(dalloc(ctx, &B->work_c, std::max<int64_t>(n_work, 1)));
    LAMB_TRY(dalloc(ctx, &B->work_i, std::max<int64_t>(n_work, 1)));
  }
  B->n_work = n_work;
  B->n_products = n_products;
  B->flops = flops;
  int64_t pos = 0;
  for (int i : B->order) {
    const int64_t m = B->sym[i].c_nnz;
    if (m) {
      LAMB_CUDA(ctx, cudaMemcpyAsync(B->work + pos, works[i], sizeof(Work) * m, cudaMemcpyDeviceToDevice, ctx->stream));
      LAMB_CUDA(ctx, cudaMemcpyAsync(B->work_c + pos, wcs[i], sizeof(int32_t) * m, cudaMemcpyDeviceToDevice, ctx->stream));
      k_fill_i32<<<grid_for(m), kThreads, 0, ctx->stream>>>(m, i, B->work_i + pos);
      LAMB_LAUNCHED(ctx);
    }
    pos += m;
  }
  if (!B->inst) LAMB_TRY(dalloc(ctx, &B->inst, std::max(n, 1)));
  LAMB_CUDA(ctx, cudaMemcpyAsync(B->inst, hinst.data(), sizeof(BatchInst) * n, cudaMemcpyHostToDevice, ctx->stream));
  if (B->by_shape) LAMB_TRY(sort_by_shape(B));
  for (int i = 0; i < n; ++i) {
    // the entries stay (the instance table points at them); the rest is not needed
    dfree(ctx, B->sym[i].stack_p);
    dfree(ctx, B->sym[i].c_row);
  }
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return LAMB_GPU_OK;
}

static void record_gens(Batch* B) {
  B->gens.clear();
  for (lamb_gpu_matrix h : B->handles) B->gens.push_back(find_matrix(B->ctx, h)->gen);
}

// One timed launch of the whole queue with cfg (after one warm-up launch).
static int32_t time_full(Batch* B, const BatchConfig& cfg, float* ms) {
  Ctx* ctx = B->ctx;
  LAMB_TRY(run_once(B, cfg, B->n_work));
  LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[5], ctx->stream));
  LAMB_TRY(run_once(B, cfg, B->n_work));
  LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[6], ctx->stream));
  LAMB_CUDA(ctx, cudaEventSynchronize(ctx->ev[6]));
  cudaEventElapsedTime(ms, ctx->ev[5], ctx->ev[6]);
  return LAMB_GPU_OK;
}

static int32_t create_batch(Ctx* ctx, const lamb_gpu_matrix* a, const lamb_gpu_matrix* b, const lamb_gpu_matrix* c,
                            int n, double eps, Batch* B) {
  B->ctx = ctx;
  B->eps = eps;
  for (int i = 0; i < n; ++i) {
    DevMatrix* A = get_matrix(ctx, a[i]);
    DevMatrix* Bm = get_matrix(ctx, b[i]);
    DevMatrix* C = get_matrix(ctx, c[i]);
    if (!A || !Bm || !C) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "batch: invalid handle");
    if (C == A || C == Bm) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "batch: C aliases A or B");
    for (int j = 0; j < i; ++j)
      if (B->c[j] == C) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "batch: C handles must differ");
    LAMB_TRY(check_compatible(ctx, A, Bm));
    LAMB_TRY(ensure_row_order(ctx, A));
    B->a.push_back(A);
    B->b.push_back(Bm);
    B->c.push_back(C);
  }
  B->sym.resize(n);
  B->nrm.assign(n, nullptr);
  B->nrm_cap.assign(n, 0);
  bool relayout = false;
  LAMB_TRY(build_queue(B, true, &relayout));
  LAMB_TRY(dalloc(ctx, &B->head, 1));
  for (int i = 0; i < n; ++i)
    for (lamb_gpu_matrix h : {a[i], b[i], c[i]}) B->handles.push_back(h);
  record_gens(B);
  LAMB_TRY(autotune(B));
  // queue order: instance-major against grouped by shape, whole queue, the tuned shape
  const std::string key = tune_signature(*B) + "_order";
  int order = -1;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) order = it->second.grab;
  }
  if (order < 0 && B->n_work > 0) {
    float ms_inst = 0, ms_shape = 0;
    LAMB_TRY(time_full(B, B->cfg, &ms_inst));
    LAMB_TRY(sort_by_shape(B));
    LAMB_TRY(time_full(B, B->cfg, &ms_shape));
    order = ms_shape < ms_inst ? 1 : 0;
    B->by_shape = order == 1;
    if (!B->by_shape) LAMB_TRY(build_queue(B, false, &relayout));  // back to instance-major
    record_gens(B);
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key] = BatchConfig{0, 0, order};
    store_tune_file(key, BatchConfig{0, 0, order});
  } else if (order == 1) {
    B->by_shape = true;
    LAMB_TRY(sort_by_shape(B));
  }
  return LAMB_GPU_OK;
}

// The operands' buffers are those the graph was built on.
static int32_t check_operands(Batch* B) {
  Ctx* ctx = B->ctx;
  for (size_t i = 0; i < B->handles.size(); ++i) {
    const DevMatrix* m = find_matrix(ctx, B->handles[i]);
    if (!m || m->gen != B->gens[i])
      return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS,
                  "batch: operand " + std::to_string(B->handles[i]) +
                      " was destroyed or its buffers replaced since lamb_gpu_batch_create");
  }
  return LAMB_GPU_OK;
}

static int32_t batch_run(Batch* B, uint32_t flags, lamb_gpu_mult_stats* stats) {
  Ctx* ctx = B->ctx;
  LAMB_TRY(settle(ctx));
  LAMB_TRY(check_operands(B));
  const bool full = (flags & LAMB_GPU_BATCH_FULL) != 0;
  const int64_t launches0 = ctx->launches;
  LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
  if (full) {
    bool relayout = false;
    LAMB_TRY(build_queue(B, false, &relayout));
    if (relayout && B->exec) {
      cudaGraphExecDestroy(B->exec);
      cudaGraphDestroy(B->graph);
      B->exec = nullptr;
      B->graph = nullptr;
    }
  }
  LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
  if (!B->exec) {
    LAMB_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int32_t rc = run_once(B, B->cfg, B->n_work);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    LAMB_TRY(rc);
    LAMB_CUDA(ctx, e);
    B->graph = g;
    LAMB_CUDA(ctx, cudaGraphInstantiate(&B->exec, B->graph, 0));
    LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
  } else {
    ++ctx->launches;  // the replayed graph holds one kernel of this library
  }
  LAMB_CUDA(ctx, cudaGraphLaunch(B->exec, ctx->stream));
  LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
  int64_t before = 0, after = 0;
  if (full) {
    for (size_t i = 0; i < B->c.size(); ++i) before += B->sym[i].c_nnz;
    if (B->eps > 0)
      for (size_t i = 0; i < B->c.size(); ++i) LAMB_TRY(result_filter(ctx, B->c[i], B->nrm[i], B->eps));
  }
  LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
  LAMB_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
  LAMB_TRY(settle(ctx));
  if (full) {
    for (DevMatrix* C : B->c) after += C->nnz;
    record_gens(B);
  }
  float t01 = 0, t12 = 0, t23 = 0, t03 = 0;
  cudaEventElapsedTime(&t01, ctx->ev[0], ctx->ev[1]);
  cudaEventElapsedTime(&t12, ctx->ev[1], ctx->ev[2]);
  cudaEventElapsedTime(&t23, ctx->ev[2], ctx->ev[3]);
  cudaEventElapsedTime(&t03, ctx->ev[0], ctx->ev[3]);
  if (stats) {
    *stats = lamb_gpu_mult_stats{};
    stats->n_products = B->n_products;
    stats->n_c_blocks = full ? after : B->n_work;
    stats->n_c_blocks_dropped = full ? before - after : 0;
    stats->flops = B->flops;
    stats->ms_symbolic = full ? t01 : 0.0;
    stats->ms_numeric = t12;
    stats->ms_filter = full ? t23 : 0.0;
    stats->ms_total = full ? t03 : t12;
    stats->kernel_launches = (int32_t)(ctx->launches - launches0);
  }
  return LAMB_GPU_OK;
}

}  // namespace lamb

using namespace lamb;

extern "C" {

int32_t lamb_gpu_batch_create(lamb_gpu_ctx* c, const lamb_gpu_matrix* a, const lamb_gpu_matrix* b,
                              const lamb_gpu_matrix* cm, int32_t n, double eps, lamb_gpu_batch** out) {
  auto* ctx = reinterpret_cast<Ctx*>(c);
  if (!ctx || !out) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  *out = nullptr;
  if (n <= 0 || !a || !b || !cm) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "batch: empty");
  cudaSetDevice(ctx->device);
  auto* B = new Batch;
  int32_t rc = create_batch(ctx, a, b, cm, n, eps, B);
  if (rc != LAMB_GPU_OK) {
    destroy_batch(B);
    return rc;
  }
  *out = reinterpret_cast<lamb_gpu_batch*>(B);
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_batch_execute(lamb_gpu_batch* bh, lamb_gpu_mult_stats* stats) {
  return lamb_gpu_batch_run(bh, 0u, stats);
}

int32_t lamb_gpu_batch_run(lamb_gpu_batch* bh, uint32_t flags, lamb_gpu_mult_stats* stats) {
  auto* B = reinterpret_cast<Batch*>(bh);
  if (!B) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  cudaSetDevice(B->ctx->device);
  return batch_run(B, flags, stats);
}

int32_t lamb_gpu_batch_queue_order(const lamb_gpu_batch* bh, int32_t* by_shape) {
  auto* B = reinterpret_cast<const Batch*>(bh);
  if (!B || !by_shape) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  *by_shape = B->by_shape ? 1 : 0;
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_batch_config(const lamb_gpu_batch* bh, int32_t* warps, int32_t* cap, int32_t* grab) {
  auto* B = reinterpret_cast<const Batch*>(bh);
  if (!B || !warps || !cap || !grab) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  *warps = B->cfg.warps;
  *cap = B->cfg.cap;
  *grab = B->cfg.grab;
  return LAMB_GPU_OK;
}

int32_t lamb_gpu_batch_destroy(lamb_gpu_batch* bh) {
  auto* B = reinterpret_cast<Batch*>(bh);
  if (!B) return LAMB_GPU_OK;
  cudaSetDevice(B->ctx->device);
  destroy_batch(B);
  return LAMB_GPU_OK;
}

}  // extern "C"
