// Charge equilibration for callers that cannot allocate device memory.
//
// Some callers own every byte of device memory themselves: a host code with its own pooled allocator and a fixed
// memory budget (a serving loop that admits work by measured bytes, a framework whose allocator must see every
// allocation), or code that runs where a device allocation and the implicit synchronisation it brings are not
// allowed. rx_qeq_solve_static gives them the charge solve of rx_qeq_solve without any allocation: the caller passes
// the matrix and every input and output as device arrays; the CG work vectors live in one file-scope device array of
// fixed size that the library reserves on every GPU that loads it, for as long as the process runs.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/rxcuda.h"

namespace rx {
namespace {

constexpr int kStaticMaxAtoms = RX_QEQ_STATIC_MAX_ATOMS;
constexpr int kMaxDevices = 64;

}  // namespace

// CG work vectors r, d, p, q for the s and t systems: 8 doubles per atom (2 MiB for 32768 atoms).
static __device__ __align__(256) double rx_qeq_static_scratch[static_cast<size_t>(kStaticMaxAtoms) * 8];

namespace {

std::mutex g_mu;
double* g_scratch[kMaxDevices] = {};

void put_err(char* err, int errlen, const char* msg) {
  if (err && errlen > 0) std::snprintf(err, static_cast<size_t>(errlen), "%s", msg);
}

__device__ inline double2 csr_row_mv(int i, const int* rs, const int* col, const double* val, double eta, const double2* v) {
  const int lane = threadIdx.x & 31;
  double ys = 0.0, yt = 0.0;
  for (int e = rs[i] + lane; e < rs[i + 1]; e += 32) {
    const double h = val[e];
    const double2 vj = v[col[e]];
    ys += h * vj.x;
    yt += h * vj.y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    ys += __shfl_xor_sync(0xffffffffu, ys, o);
    yt += __shfl_xor_sync(0xffffffffu, yt, o);
  }
  const double2 vi = v[i];
  return make_double2(eta * vi.x + __shfl_sync(0xffffffffu, ys, 0), eta * vi.y + __shfl_sync(0xffffffffu, yt, 0));
}

// A single-block Jacobi-PCG for one system held as a CSR matrix: solves
// (diag(eta) + H) s = -chi and (diag(eta) + H) t = -1 with the stopping rule of the stock fix (sqrt(r.M^-1 r)/|b| <=
// tol, at most imax - 1 iterations per system), then q = s - (sum s / sum t) t. Every work vector is written before
// it is read, so the previous call's contents of the scratch array never reach the result. A breakdown (a step length
// that is not finite, e.g. a singular or indefinite matrix) stops the loop and is reported as iters = -1 for the
// right-hand side(s) it hit.
__global__ void k_cg_csr_static(int n, const int* rs, const int* col, const double* val, const double* eta, const double* chi,
                                double* s_io, double* t_io, double* q_out, double tol, int imax, int* iters, double* rel,
                                double* scratch) {
  double2* r = reinterpret_cast<double2*>(scratch);
  double2* d = r + n;
  double2* p = d + n;
  double2* qv = p + n;
  __shared__ double sh[32 * 4];
  __shared__ double tot[4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  auto reduce = [&](double* v, int nv) {
    for (int k = 0; k < nv; ++k) {
      double x = v[k];
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) sh[wid * 4 + k] = x;
    }
    __syncthreads();
    if (threadIdx.x < nv) {
      double t = 0.0;
      for (int w = 0; w < nw; ++w) t += sh[w * 4 + threadIdx.x];
      tot[threadIdx.x] = t;
    }
    __syncthreads();
    for (int k = 0; k < nv; ++k) v[k] = tot[k];
    __syncthreads();
  };
  // the current iterate lives in d for the first product: copy the caller's guesses there
  for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = make_double2(s_io[i], t_io[i]);
  __syncthreads();
  double loc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = wid; i < n; i += nw) {
    const double e = eta[i];
    const double2 y = csr_row_mv(i, rs, col, val, e, d);
    if (lane == 0) {
      const double2 b = make_double2(-chi[i], -1.0);
      const double2 rr = make_double2(b.x - y.x, b.y - y.y);
      r[i] = rr;
      p[i] = make_double2(rr.x / e, rr.y / e);
      loc[0] += b.x * b.x; loc[1] += b.y * b.y; loc[2] += rr.x * (rr.x / e); loc[3] += rr.y * (rr.y / e);
    }
  }
  reduce(loc, 4);
  // x = guesses (kept in the caller's arrays), d = M^-1 r
  for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = p[i];
  __syncthreads();
  const double bnorm_s = sqrt(loc[0]), bnorm_t = sqrt(loc[1]);
  double sig_s = loc[2], sig_t = loc[3];
  bool act_s = true, act_t = true, broke_s = false, broke_t = false;
  int it_s = 1, it_t = 1;
  for (int it = 1; it < imax; ++it) {
    act_s = act_s && (sqrt(sig_s) / bnorm_s > tol);
    act_t = act_t && (sqrt(sig_t) / bnorm_t > tol);
    if (!act_s && !act_t) break;
    loc[0] = loc[1] = 0.0;
    for (int i = wid; i < n; i += nw) {
      const double2 y = csr_row_mv(i, rs, col, val, eta[i], d);
      if (lane == 0) {
        qv[i] = y;
        const double2 dd = d[i];
        loc[0] += dd.x * y.x; loc[1] += dd.y * y.y;
      }
    }
    reduce(loc, 2);
    const double alpha_s = act_s ? sig_s / loc[0] : 0.0;
    const double alpha_t = act_t ? sig_t / loc[1] : 0.0;
    if (!(isfinite(alpha_s) && isfinite(alpha_t))) {
      broke_s = !isfinite(alpha_s);
      broke_t = !isfinite(alpha_t);
      break;
    }
    loc[0] = loc[1] = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const double2 dd = d[i], qq = qv[i];
      double2 rr = r[i];
      s_io[i] += alpha_s * dd.x;
      t_io[i] += alpha_t * dd.y;
      rr.x -= alpha_s * qq.x; rr.y -= alpha_t * qq.y;
      r[i] = rr;
      const double e = eta[i];
      const double2 pp = make_double2(rr.x / e, rr.y / e);
      p[i] = pp;
      loc[0] += rr.x * pp.x; loc[1] += rr.y * pp.y;
    }
    reduce(loc, 2);
    const double beta_s = act_s ? loc[0] / sig_s : 0.0;
    const double beta_t = act_t ? loc[1] / sig_t : 0.0;
    if (act_s) { sig_s = loc[0]; it_s = it + 1; }
    if (act_t) { sig_t = loc[1]; it_t = it + 1; }
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const double2 pp = p[i];
      double2 dd = d[i];
      if (act_s) dd.x = pp.x + beta_s * dd.x;
      if (act_t) dd.y = pp.y + beta_t * dd.y;
      d[i] = dd;
    }
    __syncthreads();
  }
  loc[0] = loc[1] = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) { loc[0] += s_io[i]; loc[1] += t_io[i]; }
  reduce(loc, 2);
  const double u = loc[0] / loc[1];
  for (int i = threadIdx.x; i < n; i += blockDim.x) q_out[i] = s_io[i] - u * t_io[i];
  if (threadIdx.x == 0) {
    if (iters) { iters[0] = broke_s ? -1 : it_s; iters[1] = broke_t ? -1 : it_t; }
    if (rel) { rel[0] = sqrt(sig_s) / bnorm_s; rel[1] = sqrt(sig_t) / bnorm_t; }
  }
}

}  // namespace
}  // namespace rx

extern "C" int rx_qeq_solve_static(int n, const int* row_start, const int* col, const double* val, const double* eta,
                                   const double* chi, double* s, double* t, double* q, double tol, int imax, int* iters,
                                   double* rel, void* stream, char* err, int errlen) {
  using namespace rx;
  if (n < 0 || n > kStaticMaxAtoms) {
    char m[160];
    std::snprintf(m, sizeof m, "rx_qeq_solve_static: %d atoms; this entry point takes 0 (set-up only) to %d atoms (its fixed work array)", n,
                  kStaticMaxAtoms);
    put_err(err, errlen, m);
    return RX_ERR_INVALID;
  }
  if (n > 0 && (!row_start || !col || !val || !eta || !chi || !s || !t || !q)) {
    put_err(err, errlen, "rx_qeq_solve_static: null device array");
    return RX_ERR_INVALID;
  }
  if (n > 0 && (!(tol > 0.0) || imax < 1)) {
    put_err(err, errlen, "rx_qeq_solve_static: need tol > 0 and imax >= 1");
    return RX_ERR_INVALID;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    put_err(err, errlen, "rx_qeq_solve_static: no current CUDA device");
    return RX_ERR_CUDA;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch[dev]) {
      // the device address of the work array on this (current) device; the host-side name is not one. Looking it up
      // loads this library's device code on the device (with the array) if lazy module loading has not done so yet;
      // the kernel's attributes are queried too, so that its first launch loads nothing more.
      void* ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&ptr, rx_qeq_static_scratch);
      cudaFuncAttributes fa;
      if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_cg_csr_static);
      if (e != cudaSuccess) {
        char m[200];
        std::snprintf(m, sizeof m, "rx_qeq_solve_static: set-up on device %d failed: %s", dev, cudaGetErrorString(e));
        put_err(err, errlen, m);
        return RX_ERR_CUDA;
      }
      g_scratch[dev] = static_cast<double*>(ptr);
    }
    scratch = g_scratch[dev];
  }
  if (n == 0) {   // set-up only
    put_err(err, errlen, "");
    return RX_OK;
  }
  k_cg_csr_static<<<1, 512, 0, static_cast<cudaStream_t>(stream)>>>(n, row_start, col, val, eta, chi, s, t, q, tol, imax, iters,
                                                                     rel, scratch);
  // peek, not get: the error state is left as it is for the caller (an error still pending from earlier work on this
  // thread is therefore reported here too)
  const cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) {
    char m[200];
    std::snprintf(m, sizeof m, "rx_qeq_solve_static: launch failed: %s", cudaGetErrorString(e));
    put_err(err, errlen, m);
    return RX_ERR_CUDA;
  }
  put_err(err, errlen, "");
  return RX_OK;
}
