// C ABI: batched overlap SPD solves (one persistent launch replayed from a
// CUDA graph), batched / single Jacobi eigensolves, batched assembly.
#include <algorithm>
#include <mutex>
#include <numeric>
#include <vector>

#include "hp_runtime.cuh"
#include "kernels.cuh"

namespace hp {
namespace {

// Largest-n-first queue order and the batch's largest n.
void lpt_order(int count, const int64_t* off, std::vector<int>& order, int* nmax) {
  order.resize(count);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return off[a + 1] - off[a] > off[b + 1] - off[b]; });
  *nmax = 0;
  for (int i = 0; i < count; i++) *nmax = std::max<int>(*nmax, (int)(off[i + 1] - off[i]));
}

// One cached graph: the batched launch for one argument set.
struct GraphCache {
  std::mutex mu;
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  std::vector<const void*> key;
  void* order_dev = nullptr;
  void* off_dev = nullptr;
  void* work = nullptr;
  void* queue = nullptr;
};
GraphCache g_cache;

}  // namespace
}  // namespace hp

extern "C" {

int hp_spd_solve_batched_dev(int count, const int64_t* offsets, const double* centers, const double* alpha,
                             const double* b, double* x, int32_t* status, int32_t* iters, double tol, int max_iter,
                             void* stream) {
  using namespace hp;
  if (count <= 0) return count == 0 ? HP_OK : HP_ERR_INVALID_ARG;
  if (!offsets || !centers || !alpha || !b || !x || !status || !iters) return HP_ERR_INVALID_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  std::lock_guard<std::mutex> lk(g_cache.mu);
  std::vector<const void*> key = {offsets, centers, alpha, b, x, status, iters, stream,
                                  (const void*)(intptr_t)count, (const void*)(intptr_t)max_iter,
                                  (const void*)(intptr_t)(tol * 1e30)};
  // offsets is a host array: its contents are part of the key
  for (int i = 0; i <= count; i += std::max(1, count / 64)) key.push_back((const void*)(intptr_t)offsets[i]);
  key.push_back((const void*)(intptr_t)offsets[count]);
  if (g_cache.exec && key == g_cache.key) {
    HP_CUDA_TRY(cudaGraphLaunch(g_cache.exec, s));
    return HP_OK;
  }
  if (g_cache.exec) {
    cudaGraphExecDestroy(g_cache.exec);
    cudaGraphDestroy(g_cache.graph);
    cudaFree(g_cache.order_dev);
    cudaFree(g_cache.off_dev);
    cudaFree(g_cache.work);
    cudaFree(g_cache.queue);
    g_cache.exec = nullptr;
  }
  std::vector<int> order;
  int nmax = 0;
  lpt_order(count, offsets, order, &nmax);
  HP_CUDA_TRY(cudaMalloc(&g_cache.order_dev, count * sizeof(int)));
  HP_CUDA_TRY(cudaMalloc(&g_cache.off_dev, (count + 1) * sizeof(int64_t)));
  HP_CUDA_TRY(cudaMemcpy(g_cache.order_dev, order.data(), count * sizeof(int), cudaMemcpyHostToDevice));
  HP_CUDA_TRY(cudaMemcpy(g_cache.off_dev, offsets, (count + 1) * sizeof(int64_t), cudaMemcpyHostToDevice));
  // The workspace belongs to the cached graph (allocated here, outside the
  // capture); the graph holds only the queue reset and the persistent kernel.
  const int grid = batched_spd_grid(0);
  HP_CUDA_TRY(cudaMalloc(&g_cache.work, batched_spd_work_bytes(grid, nmax)));
  HP_CUDA_TRY(cudaMalloc(&g_cache.queue, sizeof(int)));
  cudaStream_t cap;
  HP_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  HP_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
  int rc = batched_spd_launch(count, (const int*)g_cache.order_dev, (const int64_t*)g_cache.off_dev, centers, alpha,
                              b, x, status, iters, nmax, tol, max_iter, g_cache.work, (int*)g_cache.queue, grid, cap);
  cudaGraph_t graph = nullptr;
  cudaError_t ce = cudaStreamEndCapture(cap, &graph);
  cudaStreamDestroy(cap);
  if (rc != HP_OK) return rc;
  if (ce != cudaSuccess) {
    set_error("batched: graph capture failed: %s", cudaGetErrorString(ce));
    return HP_ERR_CUDA;
  }
  HP_CUDA_TRY(cudaGraphInstantiate(&g_cache.exec, graph, 0));
  g_cache.graph = graph;
  g_cache.key = key;
  HP_CUDA_TRY(cudaGraphLaunch(g_cache.exec, s));
  return HP_OK;
}

int hp_spd_solve_batched(int count, const int64_t* offsets, const double* centers, const double* alpha,
                         const double* b, double* x, int32_t* status, int32_t* iters, double tol, int max_iter) {
  using namespace hp;
  if (count <= 0) return count == 0 ? HP_OK : HP_ERR_INVALID_ARG;
  if (!offsets || !centers || !alpha || !b || !x || !status || !iters) return HP_ERR_INVALID_ARG;
  const size_t N = (size_t)offsets[count];
  cudaStream_t s = library_stream();
  DevBuf dc(N * 24, s), da(N * 8, s), db(N * 16, s), dx(N * 16, s), dst(count * 4, s), dit(count * 4, s);
  if (!dc.p || !da.p || !db.p || !dx.p || !dst.p || !dit.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dc.p, centers, N * 24, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(da.p, alpha, N * 8, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(db.p, b, N * 16, cudaMemcpyHostToDevice, s));
  std::vector<int> order;
  int nmax = 0;
  lpt_order(count, offsets, order, &nmax);
  DevBuf dord(count * sizeof(int), s), doff((count + 1) * sizeof(int64_t), s);
  if (!dord.p || !doff.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dord.p, order.data(), count * sizeof(int), cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(doff.p, offsets, (count + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
  HP_TRY(batched_spd(count, dord.as<int>(), doff.as<int64_t>(), dc.as<double>(), da.as<double>(), db.as<double>(),
                     dx.as<double>(), dst.as<int>(), dit.as<int>(), nmax, tol, max_iter, s, 0));
  HP_CUDA_TRY(cudaMemcpyAsync(x, dx.p, N * 16, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaMemcpyAsync(status, dst.p, count * 4, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaMemcpyAsync(iters, dit.p, count * 4, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

int hp_overlap_norm_dd_batched_dev(int count, const int64_t* offsets, const double* centers, const double* alpha,
                                   double* S, void* stream) {
  using namespace hp;
  if (count <= 0) return count == 0 ? HP_OK : HP_ERR_INVALID_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<int64_t> mat(count);
  int64_t acc = 0;
  for (int i = 0; i < count; i++) {
    mat[i] = acc;
    const int64_t n = offsets[i + 1] - offsets[i];
    acc += n * n;
  }
  DevBuf doff((count + 1) * 8, s), dmat(count * 8, s);
  if (!doff.p || !dmat.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(doff.p, offsets, (count + 1) * 8, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dmat.p, mat.data(), count * 8, cudaMemcpyHostToDevice, s));
  HP_TRY(batched_assemble(count, doff.as<int64_t>(), centers, alpha, dmat.as<int64_t>(), S, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));  // host arrays above are freed on return
  return HP_OK;
}

int hp_f128_jacobi_eigen_batched_dev(int count, const int64_t* n_off, const double* A, size_t max_iter,
                                     double* evals, double* evecs, int32_t* sweeps, int32_t* status, void* stream) {
  using namespace hp;
  if (count <= 0) return count == 0 ? HP_OK : HP_ERR_INVALID_ARG;
  if (!n_off || !A || !evals || !evecs || !sweeps || !status) return HP_ERR_INVALID_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<int64_t> mat(count);
  int64_t acc = 0;
  int nmax = 0;
  for (int i = 0; i < count; i++) {
    mat[i] = acc;
    const int64_t n = n_off[i + 1] - n_off[i];
    acc += n * n;
    nmax = std::max<int>(nmax, (int)n);
  }
  DevBuf doff((count + 1) * 8, s), dmat(count * 8, s);
  if (!doff.p || !dmat.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(doff.p, n_off, (count + 1) * 8, cudaMemcpyHostToDevice, s));
  HP_CUDA_TRY(cudaMemcpyAsync(dmat.p, mat.data(), count * 8, cudaMemcpyHostToDevice, s));
  HP_TRY(batched_jacobi(count, doff.as<int64_t>(), dmat.as<int64_t>(), A, evals, evecs, sweeps, status, nmax,
                        (int)std::min<size_t>(max_iter, 1 << 30), s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  return HP_OK;
}

int hp_f128_jacobi_eigen(const double* a, size_t n, size_t max_iter, double* evals, double* evecs,
                         size_t* sweeps) {
  using namespace hp;
  if (n == 0) return HP_OK;
  if (!a || !evals || !evecs) return HP_ERR_INVALID_ARG;
  cudaStream_t s = library_stream();
  DevBuf dA(n * n * 16, s), dv(n * 16, s), dV(n * n * 16, s), dsw(8, s);
  if (!dA.p || !dv.p || !dV.p || !dsw.p) return HP_ERR_CUDA;
  HP_CUDA_TRY(cudaMemcpyAsync(dA.p, a, n * n * 16, cudaMemcpyHostToDevice, s));
  int64_t noff[2] = {0, (int64_t)n};
  int32_t* dsweeps = dsw.as<int32_t>();
  HP_TRY(hp_f128_jacobi_eigen_batched_dev(1, noff, dA.as<double>(), max_iter, dv.as<double>(), dV.as<double>(),
                                          dsweeps, dsweeps + 1, s));
  int32_t h[2];
  HP_CUDA_TRY(cudaMemcpyAsync(h, dsw.p, 8, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaMemcpyAsync(evals, dv.p, n * 16, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaMemcpyAsync(evecs, dV.p, n * n * 16, cudaMemcpyDeviceToHost, s));
  HP_CUDA_TRY(cudaStreamSynchronize(s));
  if (sweeps) *sweeps = (size_t)h[0];
  if (h[1] != HP_OK) {
    set_error("Jacobi eigenvalue solver did not converge within max iterations");
    return HP_ERR_NO_CONVERGE;
  }
  return HP_OK;
}

}  // extern "C"
