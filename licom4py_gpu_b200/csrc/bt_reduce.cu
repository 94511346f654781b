// bt_reduce.cu - on-device interior statistics and conservation sums.
//
// * bt_interior_stats: max, min and mean of a field's interior cells, the
//   global diagnostic of src/licom/mymodule/diag.py:45-75 computed where the
//   data lives (the reference copies the whole state to the host).
// * bt_conservation: total mass sum(h * da) and energy
//   sum((g h^2 / 2 + (H + h) |u|^2 / 2) * da) over the interior, where |u|^2 is
//   taken from the lon/lat components (a_c2l . (u, v)).  Each term is formed in
//   the field's precision; the sums are accumulated in float64 with Neumaier
//   compensation per thread and combined by a fixed binary tree, so the result
//   is deterministic and independent of launch timing.
//
// One CTA of 1024 threads walks all 6 N^2 interior cells in a fixed order; no
// scratch memory is used.

#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "bt_launch.cuh"
#include "licom_bt.h"

namespace bt {
namespace {

constexpr int kRedThreads = 1024;

struct Kahan {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double x) {  // Neumaier's variant
    const double t = s + x;
    c += (fabs(s) >= fabs(x)) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ void add(const Kahan& o) {
    add(o.s);
    c += o.c;
  }
  __device__ __forceinline__ double value() const { return s + c; }
};

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_stats(int n, const T* F, double* out) {
  const int m = n + 6, total = 6 * n * n;
  double mx = -INFINITY, mn = INFINITY;
  Kahan sum;
  for (int k = threadIdx.x; k < total; k += kRedThreads) {
    const int f = k / (n * n), r = k - f * n * n, i = r / n, j = r - i * n;
    const double v = (double)F[cell(f, i + kHalo, j + kHalo, m)];
    mx = fmax(mx, v);
    mn = fmin(mn, v);
    sum.add(v);
  }
  __shared__ double s_mx[kRedThreads], s_mn[kRedThreads], s_s[kRedThreads], s_c[kRedThreads];
  s_mx[threadIdx.x] = mx;
  s_mn[threadIdx.x] = mn;
  s_s[threadIdx.x] = sum.s;
  s_c[threadIdx.x] = sum.c;
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s_mx[threadIdx.x] = fmax(s_mx[threadIdx.x], s_mx[threadIdx.x + w]);
      s_mn[threadIdx.x] = fmin(s_mn[threadIdx.x], s_mn[threadIdx.x + w]);
      Kahan a{s_s[threadIdx.x], s_c[threadIdx.x]}, b{s_s[threadIdx.x + w], s_c[threadIdx.x + w]};
      a.add(b);
      s_s[threadIdx.x] = a.s;
      s_c[threadIdx.x] = a.c;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = s_mx[0];
    out[1] = s_mn[0];
    out[2] = (s_s[0] + s_c[0]) / (double)total;
  }
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_conservation(int n, const T* H, const T* U, const T* V,
                                                            const T* rda, const T* c2l, double depth,
                                                            double* out) {
  const int m = n + 6, total = 6 * n * n;
  Kahan mass, energy;
  for (int k = threadIdx.x; k < total; k += kRedThreads) {
    const int f = k / (n * n), r = k - f * n * n, i = r / n, j = r - i * n;
    const long o = cell(f, i + kHalo, j + kHalo, m);
    const T da = T(1.0) / rda[o];
    const T h = H[o], u = U[o], v = V[o];
    const T* C = c2l + 4 * o;
    const T ul = C[0] * u + C[1] * v, vl = C[2] * u + C[3] * v;
    mass.add((double)(h * da));
    const T e = (T(0.5) * T(9.8) * h * h + T(0.5) * (T(depth) + h) * (ul * ul + vl * vl)) * da;
    energy.add((double)e);
  }
  __shared__ double s_m[kRedThreads], s_mc[kRedThreads], s_e[kRedThreads], s_ec[kRedThreads];
  s_m[threadIdx.x] = mass.s;
  s_mc[threadIdx.x] = mass.c;
  s_e[threadIdx.x] = energy.s;
  s_ec[threadIdx.x] = energy.c;
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      Kahan a{s_m[threadIdx.x], s_mc[threadIdx.x]}, b{s_m[threadIdx.x + w], s_mc[threadIdx.x + w]};
      a.add(b);
      s_m[threadIdx.x] = a.s;
      s_mc[threadIdx.x] = a.c;
      Kahan c{s_e[threadIdx.x], s_ec[threadIdx.x]}, d{s_e[threadIdx.x + w], s_ec[threadIdx.x + w]};
      c.add(d);
      s_e[threadIdx.x] = c.s;
      s_ec[threadIdx.x] = c.c;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = s_m[0] + s_mc[0];
    out[1] = s_e[0] + s_ec[0];
  }
}

int rfail(int code, const std::string& msg) { return set_error(code, msg); }

}  // namespace
}  // namespace bt

using namespace bt;

extern "C" {

int bt_interior_stats(int n, int dtype, const void* field, void* out3, void* stream) {
  if (n < 1 || !field || !out3) return rfail(BT_EINVAL, "bt_interior_stats: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == BT_F64)
    k_stats<double><<<1, kRedThreads, 0, s>>>(n, (const double*)field, (double*)out3);
  else if (dtype == BT_F32)
    k_stats<float><<<1, kRedThreads, 0, s>>>(n, (const float*)field, (double*)out3);
  else
    return rfail(BT_EINVAL, "bt_interior_stats: dtype must be BT_F64 or BT_F32");
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rfail(BT_ECUDA, std::string("bt_interior_stats: ") + cudaGetErrorString(e));
  return BT_OK;
}

int bt_conservation(int n, int dtype, const void* h, const void* u, const void* v, const void* rda,
                    const void* a_c2l, double depth, void* out2, void* stream) {
  if (n < 1 || !h || !u || !v || !rda || !a_c2l || !out2) return rfail(BT_EINVAL, "bt_conservation: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == BT_F64)
    k_conservation<double><<<1, kRedThreads, 0, s>>>(n, (const double*)h, (const double*)u, (const double*)v,
                                                     (const double*)rda, (const double*)a_c2l, depth, (double*)out2);
  else if (dtype == BT_F32)
    k_conservation<float><<<1, kRedThreads, 0, s>>>(n, (const float*)h, (const float*)u, (const float*)v,
                                                    (const float*)rda, (const float*)a_c2l, depth, (double*)out2);
  else
    return rfail(BT_EINVAL, "bt_conservation: dtype must be BT_F64 or BT_F32");
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rfail(BT_ECUDA, std::string("bt_conservation: ") + cudaGetErrorString(e));
  return BT_OK;
}

}  // extern "C"
