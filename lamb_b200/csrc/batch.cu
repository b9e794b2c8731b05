// Batched multiplication: many independent C_b = A_b . B_b (FP64) in one
// persistent launch over a global work queue, replayed from a captured CUDA
// graph, with the launch shape picked by an autotuner.  No reference
// counterpart (the reference multiplies one matrix pair per call).
//
// Creation runs the symbolic phase of every instance (C patterns, stacks,
// work lists) with the current values: the product-filter decisions are
// frozen there, and executions recompute the numeric phase only.  The C
// handles belong to the batch until it is destroyed (their device buffers
// are baked into the graph).
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
  std::vector<DevMatrix*> c;
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
  dfree(ctx, B->work);
  dfree(ctx, B->work_c);
  dfree(ctx, B->work_i);
  dfree(ctx, B->inst);
  dfree(ctx, B->head);
  cudaStreamSynchronize(ctx->stream);
  delete B;
}

static int32_t create_batch(Ctx* ctx, const lamb_gpu_matrix* a, const lamb_gpu_matrix* b, const lamb_gpu_matrix* c,
                            int n, double eps, Batch* B) {
  B->ctx = ctx;
  std::vector<DevMatrix*> A(n), Bm(n);
  for (int i = 0; i < n; ++i) {
    A[i] = get_matrix(ctx, a[i]);
    Bm[i] = get_matrix(ctx, b[i]);
    DevMatrix* C = get_matrix(ctx, c[i]);
    if (!A[i] || !Bm[i] || !C) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "batch: invalid handle");
    if (C == A[i] || C == Bm[i]) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "batch: C aliases A or B");
    for (int j = 0; j < i; ++j)
      if (B->c[j] == C) return fail(ctx, LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS, "batch: C handles must differ");
    B->c.push_back(C);
  }
  B->sym.resize(n);
  std::vector<Work*> works(n, nullptr);
  std::vector<int32_t*> wcs(n, nullptr);
  std::vector<BatchInst> hinst(n);
  const bool filt = eps > 0;
  for (int i = 0; i < n; ++i) {
    int64_t* a_offk = nullptr;
    LAMB_TRY(check_compatible(ctx, A[i], Bm[i]));
    LAMB_TRY(ensure_row_order(ctx, A[i]));
    LAMB_TRY(pack_offk(ctx, A[i], true, &a_offk));
    int32_t rc = symbolic_phase(ctx, A[i], Bm[i], B->c[i], eps, filt, false, a_offk, &B->sym[i]);
    dfree(ctx, a_offk);
    LAMB_TRY(rc);
    LAMB_TRY(build_work(ctx, B->c[i], B->sym[i], A[i], &works[i], &wcs[i]));
    B->n_work += B->sym[i].c_nnz;
    B->n_products += B->sym[i].n_ent;
    B->flops += B->sym[i].flops;
    B->max_inner = std::max(B->max_inner, max_block(A[i]->h_col_bs));
    hinst[i] = BatchInst{B->sym[i].ent, A[i]->data, Bm[i]->data, B->c[i]->data, nullptr};
    B->c[i]->norms_valid = false;
  }
  // global queue: largest instances first (shorter tail), each instance contiguous
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return B->sym[x].flops > B->sym[y].flops; });
  LAMB_TRY(dalloc(ctx, &B->work, std::max<int64_t>(B->n_work, 1)));
  LAMB_TRY(dalloc(ctx, &B->work_c, std::max<int64_t>(B->n_work, 1)));
  LAMB_TRY(dalloc(ctx, &B->work_i, std::max<int64_t>(B->n_work, 1)));
  std::vector<int32_t> hi;
  int64_t pos = 0;
  for (int i : order) {
    const int64_t m = B->sym[i].c_nnz;
    if (m) {
      LAMB_CUDA(ctx, cudaMemcpyAsync(B->work + pos, works[i], sizeof(Work) * m, cudaMemcpyDeviceToDevice, ctx->stream));
      LAMB_CUDA(ctx, cudaMemcpyAsync(B->work_c + pos, wcs[i], sizeof(int32_t) * m, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    hi.insert(hi.end(), (size_t)m, i);
    pos += m;
  }
  if (B->n_work)
    LAMB_CUDA(ctx, cudaMemcpyAsync(B->work_i, hi.data(), sizeof(int32_t) * B->n_work, cudaMemcpyHostToDevice, ctx->stream));
  LAMB_TRY(dalloc(ctx, &B->inst, std::max(n, 1)));
  LAMB_CUDA(ctx, cudaMemcpyAsync(B->inst, hinst.data(), sizeof(BatchInst) * n, cudaMemcpyHostToDevice, ctx->stream));
  LAMB_TRY(dalloc(ctx, &B->head, 1));
  LAMB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < n; ++i) {
    dfree(ctx, works[i]);
    dfree(ctx, wcs[i]);
    // the entries stay; the other symbolic arrays are no longer needed
    dfree(ctx, B->sym[i].stack_p);
    dfree(ctx, B->sym[i].c_row);
  }
  for (int i = 0; i < n; ++i)
    for (lamb_gpu_matrix h : {a[i], b[i], c[i]}) {
      B->handles.push_back(h);
      B->gens.push_back(find_matrix(ctx, h)->gen);
    }
  return autotune(B);
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
  auto* B = reinterpret_cast<Batch*>(bh);
  if (!B) return make_status(LAMB_LEVEL_FAILURE, LAMB_TYPE_WRONG_ARGS);
  Ctx* ctx = B->ctx;
  cudaSetDevice(ctx->device);
  LAMB_TRY(settle(ctx));
  LAMB_TRY(check_operands(B));
  const int64_t launches0 = ctx->launches;
  if (!B->exec) {
    LAMB_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int32_t rc = run_once(B, B->cfg, B->n_work);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    LAMB_TRY(rc);
    LAMB_CUDA(ctx, e);
    B->graph = g;
    LAMB_CUDA(ctx, cudaGraphInstantiate(&B->exec, B->graph, 0));
  } else {
    ++ctx->launches;  // the replayed graph holds one kernel of this library
  }
  LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[5], ctx->stream));
  LAMB_CUDA(ctx, cudaGraphLaunch(B->exec, ctx->stream));
  LAMB_CUDA(ctx, cudaEventRecord(ctx->ev[6], ctx->stream));
  LAMB_CUDA(ctx, cudaEventSynchronize(ctx->ev[6]));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev[5], ctx->ev[6]);
  if (stats) {
    *stats = lamb_gpu_mult_stats{};
    stats->n_products = B->n_products;
    stats->n_c_blocks = B->n_work;
    stats->flops = B->flops;
    stats->ms_numeric = ms;
    stats->ms_total = ms;
    stats->kernel_launches = (int32_t)(ctx->launches - launches0);
  }
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
