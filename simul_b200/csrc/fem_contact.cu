// Node-to-node penalty contact between two bodies (FP64), the force model of
// the reference's staggered static contact solve
// (backend/fea/framework/contact.py:49-273, framework/scene.py:291-359):
//
//   contact_nearest_kernel   every A-surface node's nearest B-surface node
//                            (B staged through shared memory in tiles; equal
//                            distances keep the smaller index) and distance
//   contact_penalty_kernel   pairs closer than the gap tolerance:
//                            f = penalty (gap - d) (x_a - x_b) / max(|x_a - x_b|, 1e-15)
//                            added to the A node (each A-surface node has at
//                            most one pair)
//   contact_tied_kernel      tied pairs: f = -penalty ((x_a - x_b) - offset)
//   contact_b_sum_kernel     the B-node reactions -f, added per B node in
//                            pair order (the order np.add.at adds them in)
//   contact_total_kernel     sum |f| over the A components, fixed order
//
// No atomics: the forces are bitwise reproducible.  Positions are current
// coordinates (reference + displacement) in the caller's node order.
#include <cuda_runtime.h>

#include "../../include/femb200.h"
#include "fem_internal.h"
#include "fem_reduce.cuh"

namespace femb200 {

constexpr int kContactThreads = 256;

// squared distance with separate roundings (no FMA contraction), as
// x*x + y*y + z*z evaluated left to right
__device__ __forceinline__ double dist2_rn(double dx, double dy, double dz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__global__ void __launch_bounds__(kContactThreads) contact_nearest_kernel(const double* __restrict__ pos_a,
                                                                           const int* __restrict__ surf_a, int na,
                                                                           const double* __restrict__ pos_b,
                                                                           const int* __restrict__ surf_b, int nb,
                                                                           int* near, double* dist) {
  __shared__ double sb[3][kContactThreads];
  const int i = blockIdx.x * kContactThreads + threadIdx.x;
  double ax = 0.0, ay = 0.0, az = 0.0;
  if (i < na) {
    const int n = surf_a[i];
    ax = pos_a[3 * n];
    ay = pos_a[3 * n + 1];
    az = pos_a[3 * n + 2];
  }
  double best = 0.0;
  int bj = -1;
  for (int t0 = 0; t0 < nb; t0 += kContactThreads) {
    __syncthreads();
    const int j = t0 + threadIdx.x;
    if (j < nb) {
      const int n = surf_b[j];
      sb[0][threadIdx.x] = pos_b[3 * n];
      sb[1][threadIdx.x] = pos_b[3 * n + 1];
      sb[2][threadIdx.x] = pos_b[3 * n + 2];
    }
    __syncthreads();
    const int m = min(kContactThreads, nb - t0);
    for (int k = 0; k < m; ++k) {
      const double d2 = dist2_rn(__dsub_rn(ax, sb[0][k]), __dsub_rn(ay, sb[1][k]), __dsub_rn(az, sb[2][k]));
      if (bj < 0 || d2 < best) {
        best = d2;
        bj = t0 + k;
      }
    }
  }
  if (i < na) {
    near[i] = bj;
    dist[i] = bj < 0 ? 1e300 : __dsqrt_rn(best);
  }
}

// f_i for A-surface node i (zero when not in contact); f_a[node] += f_i
__global__ void contact_penalty_kernel(const double* __restrict__ pos_a, const int* __restrict__ surf_a, int na,
                                       const double* __restrict__ pos_b, const int* __restrict__ surf_b,
                                       const int* __restrict__ near, const double* __restrict__ dist,
                                       double gap, double penalty, double* fpair, double* f_a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= na) return;
  double f[3] = {0.0, 0.0, 0.0};
  const double d = dist[i];
  if (near[i] >= 0 && d < gap) {
    const int a = surf_a[i], b = surf_b[near[i]];
    const double df[3] = {__dsub_rn(pos_a[3 * a], pos_b[3 * b]), __dsub_rn(pos_a[3 * a + 1], pos_b[3 * b + 1]),
                          __dsub_rn(pos_a[3 * a + 2], pos_b[3 * b + 2])};
    double nrm = __dsqrt_rn(dist2_rn(df[0], df[1], df[2]));
    nrm = nrm > 1e-15 ? nrm : 1e-15;
    const double mag = __dmul_rn(penalty, __dsub_rn(gap, d));
    for (int k = 0; k < 3; ++k) f[k] = __dmul_rn(mag, __ddiv_rn(df[k], nrm));
    for (int k = 0; k < 3; ++k) f_a[3 * a + k] = __dadd_rn(f_a[3 * a + k], f[k]);
  }
  for (int k = 0; k < 3; ++k) fpair[3 * i + k] = f[k];
}

// tied pair p: f = -penalty ((x_a - x_b) - offset); f_a[a] += f (pairs are
// listed with each A node at most once)
__global__ void contact_tied_kernel(const double* __restrict__ pos_a, const double* __restrict__ pos_b,
                                    const int* __restrict__ pairs, const double* __restrict__ offsets, int np,
                                    double penalty, double* fpair, double* f_a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int a = pairs[2 * p], b = pairs[2 * p + 1];
  for (int k = 0; k < 3; ++k) {
    const double dev = __dsub_rn(__dsub_rn(pos_a[3 * a + k], pos_b[3 * b + k]), offsets[3 * p + k]);
    const double f = __dmul_rn(-penalty, dev);
    fpair[3 * p + k] = f;
    f_a[3 * a + k] = __dadd_rn(f_a[3 * a + k], f);
  }
}

// f_b[node of B-surface j] -= sum over pairs with near == j of f, in pair
// order.  key[p] = the pair's B-surface index (or -1); one thread per B
// node, the pairs staged in shared memory in tiles.
__global__ void __launch_bounds__(kContactThreads) contact_b_sum_kernel(const int* __restrict__ key,
                                                                         const double* __restrict__ fpair, int np,
                                                                         const int* __restrict__ nodes_b, int nb,
                                                                         double* f_b) {
  __shared__ int sk[kContactThreads];
  __shared__ double sf[3][kContactThreads];
  const int j = blockIdx.x * kContactThreads + threadIdx.x;
  double acc[3] = {0.0, 0.0, 0.0};
  bool hit = false;
  for (int t0 = 0; t0 < np; t0 += kContactThreads) {
    __syncthreads();
    const int p = t0 + threadIdx.x;
    sk[threadIdx.x] = p < np ? key[p] : -1;
    if (p < np)
      for (int k = 0; k < 3; ++k) sf[k][threadIdx.x] = fpair[3 * p + k];
    __syncthreads();
    const int m = min(kContactThreads, np - t0);
    for (int q = 0; q < m; ++q)
      if (sk[q] == j) {
        hit = true;
        for (int k = 0; k < 3; ++k) acc[k] = __dsub_rn(acc[k], sf[k][q]);
      }
  }
  if (j < nb && hit) {
    const int n = nodes_b[j];
    for (int k = 0; k < 3; ++k) f_b[3 * n + k] = __dadd_rn(f_b[3 * n + k], acc[k]);
  }
}

// key[i] = near[i] if A-surface node i is in contact, else -1; count pairs
__global__ void contact_key_kernel(const int* __restrict__ near, const double* __restrict__ dist, int na, double gap,
                                   int* key) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= na) return;
  key[i] = (near[i] >= 0 && dist[i] < gap) ? near[i] : -1;
}

// total = sum of |f| over all pair components, and the number of pairs with
// key >= 0 (one CTA, fixed order)
__global__ void __launch_bounds__(kContactThreads) contact_total_kernel(const double* __restrict__ fpair,
                                                                         const int* __restrict__ key, int np,
                                                                         double* out) {
  __shared__ double sred[kContactThreads / 32];
  double s = 0.0, c = 0.0;
  for (int p = threadIdx.x; p < np; p += kContactThreads) {
    if (key && key[p] < 0) continue;
    c += 1.0;
    for (int k = 0; k < 3; ++k) s += fabs(fpair[3 * p + k]);
  }
  const double ts = block_sum<kContactThreads>(s, sred);
  const double tc = block_sum<kContactThreads>(c, sred);
  if (threadIdx.x == 0) {
    out[0] = ts;
    out[1] = tc;
  }
}

__global__ void contact_iota_kernel(int* out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = i;
}

}  // namespace femb200

using namespace femb200;

namespace {

inline int cblk(int n) { return (n + kContactThreads - 1) / kContactThreads; }

struct Scratch {
  void* p[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  ~Scratch() {
    for (void* q : p)
      if (q) cudaFree(q);
  }
};

}  // namespace

extern "C" {

int fem_contact_nearest(const double* pos_a, const int32_t* surf_a, int32_t na, const double* pos_b,
                        const int32_t* surf_b, int32_t nb, int32_t* nearest, double* dist, void* stream) {
  if (na < 0 || nb < 0) return set_global_error(FEM_ERR_INVALID, "negative surface size");
  if (na == 0) return FEM_OK;
  if (!pos_a || !surf_a || !pos_b || (nb > 0 && !surf_b) || !nearest || !dist)
    return set_global_error(FEM_ERR_INVALID, "null array");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  contact_nearest_kernel<<<cblk(na), kContactThreads, 0, s>>>(pos_a, surf_a, na, pos_b, surf_b, nb, nearest, dist);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_global_error(FEM_ERR_CUDA, "contact nearest: %s", cudaGetErrorString(e));
  return FEM_OK;
}

int fem_contact_penalty(const double* pos_a, const int32_t* surf_a, int32_t na, const double* pos_b,
                        const int32_t* surf_b, int32_t nb, double gap_tol, double penalty, double* f_a, double* f_b,
                        int32_t* n_pairs, double* total, void* stream) {
  if (na < 0 || nb < 0) return set_global_error(FEM_ERR_INVALID, "negative surface size");
  if (n_pairs) *n_pairs = 0;
  if (total) *total = 0.0;
  if (na == 0 || nb == 0) return FEM_OK;
  if (!pos_a || !surf_a || !pos_b || !surf_b || !f_a || !f_b) return set_global_error(FEM_ERR_INVALID, "null array");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Scratch w;
  cudaError_t e = cudaMalloc(&w.p[0], sizeof(int) * (size_t)na);
  if (e == cudaSuccess) e = cudaMalloc(&w.p[1], sizeof(double) * (size_t)na);
  if (e == cudaSuccess) e = cudaMalloc(&w.p[2], sizeof(double) * 3 * (size_t)na);
  if (e == cudaSuccess) e = cudaMalloc(&w.p[3], sizeof(int) * (size_t)na);
  if (e == cudaSuccess) e = cudaMalloc(&w.p[4], sizeof(double) * 2);
  if (e != cudaSuccess) return set_global_error(FEM_ERR_CUDA, "contact scratch: %s", cudaGetErrorString(e));
  int* near = static_cast<int*>(w.p[0]);
  double* dist = static_cast<double*>(w.p[1]);
  double* fpair = static_cast<double*>(w.p[2]);
  int* key = static_cast<int*>(w.p[3]);
  double* tot = static_cast<double*>(w.p[4]);
  contact_nearest_kernel<<<cblk(na), kContactThreads, 0, s>>>(pos_a, surf_a, na, pos_b, surf_b, nb, near, dist);
  contact_penalty_kernel<<<cblk(na), kContactThreads, 0, s>>>(pos_a, surf_a, na, pos_b, surf_b, near, dist, gap_tol,
                                                              penalty, fpair, f_a);
  contact_key_kernel<<<cblk(na), kContactThreads, 0, s>>>(near, dist, na, gap_tol, key);
  contact_b_sum_kernel<<<cblk(nb), kContactThreads, 0, s>>>(key, fpair, na, surf_b, nb, f_b);
  contact_total_kernel<<<1, kContactThreads, 0, s>>>(fpair, key, na, tot);
  double h[2] = {0.0, 0.0};
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, tot, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_global_error(FEM_ERR_CUDA, "contact penalty: %s", cudaGetErrorString(e));
  if (n_pairs) *n_pairs = (int32_t)h[1];
  if (total) *total = h[0];
  return FEM_OK;
}

int fem_contact_tied(const double* pos_a, const double* pos_b, const int32_t* pairs, const double* offsets,
                     int32_t n_pairs, int32_t nb_nodes, double penalty, double* f_a, double* f_b, double* total,
                     void* stream) {
  if (n_pairs < 0 || nb_nodes < 0) return set_global_error(FEM_ERR_INVALID, "negative size");
  if (total) *total = 0.0;
  if (n_pairs == 0) return FEM_OK;
  if (!pos_a || !pos_b || !pairs || !offsets || !f_a || !f_b) return set_global_error(FEM_ERR_INVALID, "null array");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Scratch w;
  cudaError_t e = cudaMalloc(&w.p[0], sizeof(double) * 3 * (size_t)n_pairs);
  if (e == cudaSuccess) e = cudaMalloc(&w.p[1], sizeof(int) * (size_t)n_pairs);
  if (e == cudaSuccess) e = cudaMalloc(&w.p[2], sizeof(int) * (size_t)nb_nodes);
  if (e == cudaSuccess) e = cudaMalloc(&w.p[3], sizeof(double) * 2);
  if (e != cudaSuccess) return set_global_error(FEM_ERR_CUDA, "contact scratch: %s", cudaGetErrorString(e));
  double* fpair = static_cast<double*>(w.p[0]);
  int* key = static_cast<int*>(w.p[1]);
  int* ident = static_cast<int*>(w.p[2]);
  double* tot = static_cast<double*>(w.p[3]);
  contact_tied_kernel<<<cblk(n_pairs), kContactThreads, 0, s>>>(pos_a, pos_b, pairs, offsets, n_pairs, penalty,
                                                                fpair, f_a);
  // B reactions keyed by the B node itself (identity "surface" over all B nodes)
  e = cudaMemcpy2DAsync(key, sizeof(int), pairs + 1, 2 * sizeof(int), sizeof(int), n_pairs, cudaMemcpyDeviceToDevice,
                        s);
  if (e != cudaSuccess) return set_global_error(FEM_ERR_CUDA, "contact tied: %s", cudaGetErrorString(e));
  contact_iota_kernel<<<cblk(nb_nodes), kContactThreads, 0, s>>>(ident, nb_nodes);
  contact_b_sum_kernel<<<cblk(nb_nodes), kContactThreads, 0, s>>>(key, fpair, n_pairs, ident, nb_nodes, f_b);
  contact_total_kernel<<<1, kContactThreads, 0, s>>>(fpair, nullptr, n_pairs, tot);
  double h[2] = {0.0, 0.0};
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, tot, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_global_error(FEM_ERR_CUDA, "contact tied: %s", cudaGetErrorString(e));
  if (total) *total = h[0];
  return FEM_OK;
}

}  // extern "C"
