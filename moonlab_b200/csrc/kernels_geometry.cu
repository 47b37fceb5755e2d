// kernels_geometry.cu -- Gram matrix of a batch of complex128 states in FP64,
// G[a][b] = sum_x conj(S_a[x]) S_b[x] for a <= b: the inner products the
// quantum geometric tensor is assembled from (adjoint.cpp,
// mlb_hea_geometry).
//
// The B x B upper triangle is cut into 32 x 32 tile pairs (ta <= tb); the
// amplitude axis into K chunks.  One CTA takes one (pair, chunk): it stages
// 32 amplitudes of the pair's 32 + 32 rows in shared memory per step
// (coalesced 512-byte row runs) and each of its 256 threads accumulates a
// 2 x 2 block of conj(x) y in FP64 (rows ty, ty + 16 of tile ta, columns tx,
// tx + 16 of tile tb: the 8 threads of a shared-memory phase read 8
// distinct rows, one per bank group, thanks to the 33-element row pitch).
// Per-chunk partials are then summed in chunk order by a second kernel, so
// the result does not depend on scheduling.
#include <vector>

#include "kernels_common.cuh"
#include "mlb_internal.h"

namespace mlb {

namespace {

constexpr int kGT = 32;  // rows per tile
constexpr int kGK = 32;  // amplitudes per shared-memory step

__global__ void __launch_bounds__(256) k_gram_partial(const double2* __restrict__ S, uint64_t dim, int B,
                                                      const int2* __restrict__ pairs, int npairs,
                                                      uint64_t kchunk, double2* __restrict__ part) {
  __shared__ double2 sa[kGT][kGK + 1];
  __shared__ double2 sb[kGT][kGK + 1];
  const int2 pr = pairs[blockIdx.x];
  const int a0 = pr.x * kGT, b0 = pr.y * kGT;
  const uint64_t k0 = (uint64_t)blockIdx.y * kchunk;
  const uint64_t k1 = k0 + kchunk < dim ? k0 + kchunk : dim;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double ar[2][2] = {{0.0, 0.0}, {0.0, 0.0}}, ai[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (uint64_t k = k0; k < k1; k += kGK) {
    for (int e = threadIdx.x; e < kGT * kGK; e += 256) {
      const int r = e / kGK, c = e % kGK;
      const uint64_t x = k + (uint64_t)c;
      double2 va = make_double2(0.0, 0.0), vb = make_double2(0.0, 0.0);
      if (x < k1) {
        if (a0 + r < B) va = S[(uint64_t)(a0 + r) * dim + x];
        if (b0 + r < B) vb = S[(uint64_t)(b0 + r) * dim + x];
      }
      sa[r][c] = va;
      sb[r][c] = vb;
    }
    __syncthreads();
#pragma unroll 8
    for (int c = 0; c < kGK; c++) {
      const double2 x0 = sa[ty][c], x1 = sa[ty + 16][c];
      const double2 y0 = sb[tx][c], y1 = sb[tx + 16][c];
      const double2 xs[2] = {x0, x1}, ys[2] = {y0, y1};
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) {
          ar[i][j] = fma(xs[i].x, ys[j].x, fma(xs[i].y, ys[j].y, ar[i][j]));
          ai[i][j] = fma(xs[i].x, ys[j].y, fma(-xs[i].y, ys[j].x, ai[i][j]));
        }
    }
    __syncthreads();
  }
  double2* out = part + ((size_t)blockIdx.y * npairs + blockIdx.x) * (kGT * kGT);
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++) out[(ty + 16 * i) * kGT + tx + 16 * j] = make_double2(ar[i][j], ai[i][j]);
}

// G[a][b] (a <= b, both < B) = sum over chunks, in chunk order.
__global__ void k_gram_reduce(const double2* __restrict__ part, const int2* __restrict__ pairs, int npairs,
                              int nchunks, int B, double2* __restrict__ G) {
  const int p = blockIdx.x;
  const int2 pr = pairs[p];
  for (int e = threadIdx.x; e < kGT * kGT; e += blockDim.x) {
    const int a = pr.x * kGT + e / kGT, b = pr.y * kGT + e % kGT;
    if (a >= B || b >= B || a > b) continue;
    double2 s = make_double2(0.0, 0.0);
    for (int c = 0; c < nchunks; c++) {
      const double2 v = part[((size_t)c * npairs + p) * (kGT * kGT) + e];
      s.x += v.x;
      s.y += v.y;
    }
    G[(size_t)a * B + b] = s;
  }
}

// Launch geometry of one Gram computation: tile pairs, K chunks (about four
// CTAs per SM in all) and the chunk length in amplitudes (a multiple of kGK).
struct GramGeo {
  int npairs;
  uint64_t nchunks, kchunk;
  size_t pairs_bytes;  // the pair table, padded to 256 bytes
};
GramGeo gram_geo(int B, uint64_t dim, int num_sms) {
  GramGeo g;
  const int T = (B + kGT - 1) / kGT;
  g.npairs = T * (T + 1) / 2;
  const uint64_t steps = (dim + kGK - 1) / kGK;
  uint64_t nchunks = (uint64_t)(4 * num_sms + g.npairs - 1) / (uint64_t)g.npairs;
  if (nchunks < 1) nchunks = 1;
  if (nchunks > steps) nchunks = steps;
  g.kchunk = ((steps + nchunks - 1) / nchunks) * kGK;
  g.nchunks = (dim + g.kchunk - 1) / g.kchunk;
  g.pairs_bytes = (sizeof(int2) * (size_t)g.npairs + 255) / 256 * 256;
  return g;
}

}  // namespace

size_t gram_scratch_bytes(int B, uint64_t dim, int num_sms) {
  const GramGeo g = gram_geo(B, dim, num_sms);
  return g.pairs_bytes + sizeof(double2) * (size_t)g.nchunks * g.npairs * kGT * kGT;
}

int launch_gram(const void* states, uint64_t dim, int B, double2* d_G, void* d_scratch, int num_sms,
                cudaStream_t stream) {
  if (B < 1 || dim < 1) return MLB_ERR_INVALID_ARG;
  const GramGeo g = gram_geo(B, dim, num_sms);
  const int T = (B + kGT - 1) / kGT;
  const int npairs = g.npairs;
  const uint64_t kchunk = g.kchunk, nchunks = g.nchunks;
  // tile-pair table at the start of the scratch (256-byte padded), partials after it
  int2* d_pairs = static_cast<int2*>(d_scratch);
  double2* d_part = reinterpret_cast<double2*>(static_cast<unsigned char*>(d_scratch) + g.pairs_bytes);
  std::vector<int2> pairs;
  pairs.reserve(npairs);
  for (int a = 0; a < T; a++)
    for (int b = a; b < T; b++) pairs.push_back(make_int2(a, b));
  if (cudaMemcpyAsync(d_pairs, pairs.data(), sizeof(int2) * pairs.size(), cudaMemcpyHostToDevice, stream) !=
      cudaSuccess)
    return MLB_ERR_DRIVER;
  dim3 grid((unsigned)npairs, (unsigned)nchunks);
  k_gram_partial<<<grid, 256, 0, stream>>>(static_cast<const double2*>(states), dim, B, d_pairs, npairs, kchunk,
                                           d_part);
  k_gram_reduce<<<npairs, 256, 0, stream>>>(d_part, d_pairs, npairs, (int)nchunks, B, d_G);
  count_launch(2);
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

}  // namespace mlb
