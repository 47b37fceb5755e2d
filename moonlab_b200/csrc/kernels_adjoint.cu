// kernels_adjoint.cu -- batched adjoint gradient of a hardware-efficient
// ansatz energy E(theta) = <psi(theta)|H|psi(theta)>, H a sum of Pauli strings.
//
// The reference (differentiable.c:438-491, per Hamiltonian term) walks the
// gate tape backwards once per term, cloning states and taking one inner
// product per parameter.  The gradient is linear in the observable, so here
// lambda = H psi is formed once and a single backward sweep carries (psi,
// lambda) through the inverse gates:  dE/dtheta_p = Im<lambda|G_p|psi> at the
// point where both states stand just after gate p (G = Y for RY, Z for RZ).
//
// Batch layout: B parameter vectors give B states stored back to back,
// [B][2^N]; a tile never spans two batch elements, so every tile reads the
// cos/sin of its own theta (table cs[b][p], computed once per call).
//
// Kernels (all tile passes, one HBM read + write of each array per pass):
//   k_adj_gates : gate ops on psi (forward) or on psi and lambda together
//                 with the per-parameter partial inner products (backward).
//                 Register groups of 2^3 amplitudes per thread, as in the
//                 state engine's tile passes.
//   k_adj_pauli : lambda (+)= sum_k c_k P_k psi for the Pauli terms whose
//                 X-part lies inside the tile; the last pass also emits the
//                 per-tile partial of Re<psi|lambda> (the energy).
//   k_adj_reduce: fixed-order sums of the per-tile partials (deterministic).
// Tiles come into shared memory by asynchronous copies, all in flight at
// once.  (Issuing the next tile's copies from the store loop, as the state
// engine's tile passes do, measured no faster here.)
#include <cstdio>

#include "kernels_common.cuh"
#include "mlb_internal.h"

namespace mlb {

namespace {

template <typename Real> struct AdjCfg;
template <> struct AdjCfg<double> { static constexpr int TB = 11, NT = 256, SW_SHIFT = 3, SW_MASK = 7; };
template <> struct AdjCfg<float> { static constexpr int TB = 12, NT = 256, SW_SHIFT = 4, SW_MASK = 15; };
constexpr int kRB = 3, kG = 1 << kRB;

template <typename Real>
__device__ __forceinline__ uint32_t aswz(uint32_t e) {
  return e ^ ((e >> AdjCfg<Real>::SW_SHIFT) & AdjCfg<Real>::SW_MASK);
}

__device__ __forceinline__ uint64_t tile_base_of(const AdjPass& P, uint64_t tile) {
  const uint64_t b = tile / P.tiles_per_state, t = tile % P.tiles_per_state;
  return (b << P.n) | pdep64(t, P.tile_free_mask);
}

// HBM -> shared by asynchronous copies: every load of the tile is in flight
// at once (a load-then-store loop would wait out each load's latency in
// turn).  The caller completes them with tile_loads_wait() and a barrier.
template <typename Real>
__device__ __forceinline__ void load_tile(typename Cplx<Real>::T* __restrict__ sm,
                                          const typename Cplx<Real>::T* __restrict__ g,
                                          uint64_t tile_base, const uint64_t* rowoff, int L, uint32_t amps) {
  using A = typename Cplx<Real>::T;
  constexpr int NT = AdjCfg<Real>::NT;
  const uint32_t lm = (1u << L) - 1u;
  const uint32_t base = static_cast<uint32_t>(__cvta_generic_to_shared(sm));
#pragma unroll 1
  for (uint32_t e = threadIdx.x; e < amps; e += NT) {
    const A* src = &g[tile_base | rowoff[e >> L] | (e & lm)];
    const uint32_t dst = base + aswz<Real>(e) * (uint32_t)sizeof(A);
    if constexpr (sizeof(A) == 16)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
    else
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
  }
}
__device__ __forceinline__ void tile_loads_wait() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}
template <typename Real>
__device__ __forceinline__ void store_tile(const typename Cplx<Real>::T* __restrict__ sm,
                                           typename Cplx<Real>::T* __restrict__ g, uint64_t tile_base,
                                           const uint64_t* rowoff, int L, uint32_t amps) {
  constexpr int NT = AdjCfg<Real>::NT;
  const uint32_t lm = (1u << L) - 1u;
  for (uint32_t e = threadIdx.x; e < amps; e += NT) __stcs(&g[tile_base | rowoff[e >> L] | (e & lm)], sm[aswz<Real>(e)]);
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// gate passes
// ---------------------------------------------------------------------------
template <typename A, int RT, bool DUAL>
__device__ __forceinline__ void apply_x(A (&v)[kG], A (&w)[kG], uint32_t gb, const uint32_t (&bm)[kRB],
                                        uint32_t lcmask) {
#pragma unroll
  for (int k = 0; k < kG; k++) {
    if (k & (1 << RT)) continue;
    uint32_t loc = gb;
#pragma unroll
    for (int b = 0; b < kRB; b++)
      if (k >> b & 1) loc |= bm[b];
    if ((loc & lcmask) != lcmask) continue;
    const int k1 = k | (1 << RT);
    A t = v[k]; v[k] = v[k1]; v[k1] = t;
    if (DUAL) { t = w[k]; w[k] = w[k1]; w[k1] = t; }
  }
}

// RY(angle) with c, s of the applied angle: [[c, -s], [s, c]].
template <typename A, typename Real, int RT, bool DUAL>
__device__ __forceinline__ void apply_ry(A (&v)[kG], A (&w)[kG], Real c, Real s) {
#pragma unroll
  for (int k = 0; k < kG; k++) {
    if (k & (1 << RT)) continue;
    const int k1 = k | (1 << RT);
    A a0 = v[k], a1 = v[k1];
    v[k] = {c * a0.x - s * a1.x, c * a0.y - s * a1.y};
    v[k1] = {s * a0.x + c * a1.x, s * a0.y + c * a1.y};
    if (DUAL) {
      a0 = w[k]; a1 = w[k1];
      w[k] = {c * a0.x - s * a1.x, c * a0.y - s * a1.y};
      w[k1] = {s * a0.x + c * a1.x, s * a0.y + c * a1.y};
    }
  }
}

// Im<lambda|Y_q|psi> over the pairs of register bit RT:
// (Y psi)_{q=0} = -i psi_{q=1},  (Y psi)_{q=1} = i psi_{q=0}.
template <typename A, int RT>
__device__ __forceinline__ double grad_y(const A (&v)[kG], const A (&w)[kG]) {
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < kG; k++) {
    if (k & (1 << RT)) continue;
    const int k1 = k | (1 << RT);
    const A p0 = v[k], p1 = v[k1], l0 = w[k], l1 = w[k1];
    acc += -((double)l0.x * p1.x + (double)l0.y * p1.y) + ((double)l1.x * p0.x + (double)l1.y * p0.y);
  }
  return acc;
}

template <typename Real, bool DUAL, bool BACKWARD>
__global__ void __launch_bounds__(AdjCfg<Real>::NT, 2)
    k_adj_gates(typename Cplx<Real>::T* __restrict__ psi, typename Cplx<Real>::T* __restrict__ lam,
                const AdjPass P, const AdjOp* __restrict__ ops, const double2* __restrict__ cs,
                double* __restrict__ partials) {
  using A = typename Cplx<Real>::T;
  constexpr int NT = AdjCfg<Real>::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t amps = 1u << (P.L + P.H);
  A* sv = reinterpret_cast<A*>(smem_raw);
  A* sw = sv + amps;
  __shared__ uint64_t rowoff[1 << (AdjCfg<Real>::TB - 5)];
  __shared__ AdjOp sops[kMaxAdjOps];
  __shared__ double2 scs[kMaxAdjOps];
  __shared__ uint8_t son[kMaxAdjOps];
  __shared__ double red[NT / 32][kMaxAdjSlots];

  for (uint32_t r = threadIdx.x; r < (1u << P.H); r += NT) {
    uint64_t off = 0;
#pragma unroll
    for (int k = 0; k < kMaxHigh; k++)
      if (k < P.H && (r >> k & 1u)) off |= 1ull << P.high[k];
    rowoff[r] = off;
  }
  for (int o = threadIdx.x; o < P.num_ops; o += NT) sops[o] = ops[o];
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint64_t tile = blockIdx.x; tile < P.num_tiles; tile += gridDim.x) {
    const uint64_t tb = tile_base_of(P, tile);
    const uint64_t b = tile / P.tiles_per_state;
    for (int o = threadIdx.x; o < P.num_ops; o += NT) {
      const AdjOp& op = sops[o];
      son[o] = (uint8_t)((tb & op.ocmask) == op.ocmask);
      if (op.p >= 0) scs[o] = cs[b * P.num_params + op.p];
    }
    for (int i = threadIdx.x; i < (NT / 32) * kMaxAdjSlots; i += NT) (&red[0][0])[i] = 0.0;
    load_tile<Real>(sv, psi, tb, rowoff, P.L, amps);
    if (DUAL) load_tile<Real>(sw, lam, tb, rowoff, P.L, amps);
    tile_loads_wait();
    __syncthreads();

    for (int s = 0; s < P.num_segments; s++) {
      const AdjSeg& seg = P.segs[s];
      uint32_t bm[kRB];
#pragma unroll
      for (int q = 0; q < kRB; q++) bm[q] = 1u << seg.bits[q];
      const uint32_t groups = amps >> kRB;
      // Every lane runs every iteration (the gradient partials use full-warp
      // shuffles); lanes past the last group work on zeros and store nothing.
      for (uint32_t g0 = 0; g0 < groups; g0 += NT) {
        const uint32_t gi = g0 + threadIdx.x;
        const bool active = gi < groups;
        uint32_t gb = active ? gi : 0u;
#pragma unroll
        for (int q = 0; q < kRB; q++) {
          const uint32_t p = seg.bits[q];
          gb = ((gb >> p) << (p + 1)) | (gb & ((1u << p) - 1u));
        }
        A v[kG], w[kG];
#pragma unroll
        for (int k = 0; k < kG; k++) {
          uint32_t loc = gb;
#pragma unroll
          for (int q = 0; q < kRB; q++)
            if (k >> q & 1) loc |= bm[q];
          v[k] = active ? sv[aswz<Real>(loc)] : A{0, 0};
          if (DUAL) w[k] = active ? sw[aswz<Real>(loc)] : A{0, 0};
        }
        for (int o = seg.op_begin; o < seg.op_end; o++) {
          if (!son[o]) continue;
          const AdjOp& op = sops[o];
          const Real c = (Real)scs[o].x, sn = (Real)scs[o].y;
          switch (op.kind * 4 + op.rt) {
#define ADJ_X(r)                                                          \
  case ADJ_KIND_X * 4 + r: apply_x<A, r, DUAL>(v, w, gb, bm, op.lcmask); break;
            ADJ_X(0) ADJ_X(1) ADJ_X(2)
#undef ADJ_X
#define ADJ_RY(r)                                                                         \
  case ADJ_KIND_RY * 4 + r:                                                               \
    if (BACKWARD && op.slot >= 0) {                                                       \
      const double t = warp_sum(grad_y<A, r>(v, w));                                      \
      if (lane == 0) red[warp][op.slot] += t;                                             \
    }                                                                                     \
    apply_ry<A, Real, r, DUAL>(v, w, c, BACKWARD ? -sn : sn);                             \
    break;
            ADJ_RY(0) ADJ_RY(1) ADJ_RY(2)
#undef ADJ_RY
            default: {  // RZ (diagonal): phases (c -+ i s) keyed on the target bit
              const uint32_t tkey = op.lt < 0 ? (uint32_t)((tb >> op.qt) & 1ull) : 0u;
              double gz = 0.0;
#pragma unroll
              for (int k = 0; k < kG; k++) {
                uint32_t loc = gb;
#pragma unroll
                for (int q = 0; q < kRB; q++)
                  if (k >> q & 1) loc |= bm[q];
                const uint32_t key = op.lt < 0 ? tkey : ((loc >> op.lt) & 1u);
                if (BACKWARD && op.slot >= 0)
                  gz += (key ? -1.0 : 1.0) * ((double)w[k].x * v[k].y - (double)w[k].y * v[k].x);
                // forward RZ(theta): key 0 -> c - i s, key 1 -> c + i s; backward: conjugate
                const Real si = ((key != 0) != BACKWARD) ? sn : -sn;
                const A ph = {c, si};
                v[k] = cmul(ph, v[k]);
                if (DUAL) w[k] = cmul(ph, w[k]);
              }
              if (BACKWARD && op.slot >= 0) {
                const double t = warp_sum(gz);
                if (lane == 0) red[warp][op.slot] += t;
              }
            }
          }
        }
        if (active) {
#pragma unroll
          for (int k = 0; k < kG; k++) {
            uint32_t loc = gb;
#pragma unroll
            for (int q = 0; q < kRB; q++)
              if (k >> q & 1) loc |= bm[q];
            sv[aswz<Real>(loc)] = v[k];
            if (DUAL) sw[aswz<Real>(loc)] = w[k];
          }
        }
      }
      __syncthreads();
    }
    store_tile<Real>(sv, psi, tb, rowoff, P.L, amps);
    if (DUAL) store_tile<Real>(sw, lam, tb, rowoff, P.L, amps);
    if (BACKWARD) {
      for (int j = threadIdx.x; j < P.num_slots; j += NT) {
        double t = 0.0;
        for (int wp = 0; wp < NT / 32; wp++) t += red[wp][j];
        partials[tile * P.num_slots + j] = t;
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// lambda (+)= sum_k c_k P_k psi, P_k|i> = i^{ny} (-1)^{|i & z|} |i ^ x>
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void __launch_bounds__(AdjCfg<Real>::NT, 1)
    k_adj_pauli(const typename Cplx<Real>::T* __restrict__ psi, typename Cplx<Real>::T* __restrict__ lam,
                const AdjPass P, const AdjTerm* __restrict__ terms, int accumulate, int want_energy,
                double* __restrict__ energy_partials) {
  using A = typename Cplx<Real>::T;
  constexpr int NT = AdjCfg<Real>::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t amps = 1u << (P.L + P.H);
  A* sv = reinterpret_cast<A*>(smem_raw);
  __shared__ uint64_t rowoff[1 << (AdjCfg<Real>::TB - 5)];
  __shared__ AdjTerm st[kMaxAdjTerms];
  __shared__ double red[NT / 32];
  for (uint32_t r = threadIdx.x; r < (1u << P.H); r += NT) {
    uint64_t off = 0;
#pragma unroll
    for (int k = 0; k < kMaxHigh; k++)
      if (k < P.H && (r >> k & 1u)) off |= 1ull << P.high[k];
    rowoff[r] = off;
  }
  for (int t = threadIdx.x; t < P.num_ops; t += NT) st[t] = terms[t];
  __syncthreads();
  const uint32_t lm = (1u << P.L) - 1u;
  for (uint64_t tile = blockIdx.x; tile < P.num_tiles; tile += gridDim.x) {
    const uint64_t tb = tile_base_of(P, tile);
    load_tile<Real>(sv, psi, tb, rowoff, P.L, amps);
    tile_loads_wait();
    __syncthreads();
    double e_acc = 0.0;
    for (uint32_t e = threadIdx.x; e < amps; e += NT) {
      double ax = 0.0, ay = 0.0;
      for (int t = 0; t < P.num_ops; t++) {
        const AdjTerm& T = st[t];
        const uint32_t src = e ^ T.xl;
        const A a = sv[aswz<Real>(src)];
        // sign from the source index: local part plus the tile-constant part
        const int par = (__popc(src & T.zl) + (int)__popcll(tb & T.zo)) & 1;
        const double cr = par ? -T.cr : T.cr, ci = par ? -T.ci : T.ci;
        ax += cr * a.x - ci * a.y;
        ay += cr * a.y + ci * a.x;
      }
      const uint64_t gidx = tb | rowoff[e >> P.L] | (e & lm);
      if (accumulate) {
        const A old = lam[gidx];
        ax += old.x;
        ay += old.y;
      }
      lam[gidx] = A{(Real)ax, (Real)ay};
      if (want_energy) {
        const A p = sv[aswz<Real>(e)];
        e_acc += (double)p.x * (Real)ax + (double)p.y * (Real)ay;  // Re(conj(psi) lambda)
      }
    }
    if (want_energy) {
      const double t = warp_sum(e_acc);
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
      __syncthreads();
      if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < NT / 32; w++) s += red[w];
        energy_partials[tile] = s;
      }
    }
    __syncthreads();
  }
}

// out[b * P + param_of_slot[j]] = sum over the tiles of batch element b of
// partials[tile][j], in tile order.
__global__ void k_adj_reduce(const double* __restrict__ partials, uint64_t tiles_per_state, int num_slots,
                             uint64_t batch, const int* __restrict__ param_of_slot, int num_params,
                             double* __restrict__ out) {
  const uint64_t total = batch * (uint64_t)num_slots;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = i / num_slots;
    const int j = (int)(i % num_slots);
    double s = 0.0;
    const double* p = partials + b * tiles_per_state * num_slots + j;
    for (uint64_t t = 0; t < tiles_per_state; t++) s += p[t * num_slots];
    out[b * num_params + (param_of_slot ? param_of_slot[j] : 0)] = s;
  }
}

template <typename Real>
__global__ void k_adj_init(typename Cplx<Real>::T* __restrict__ psi, uint64_t dim, uint64_t total, uint64_t hf) {
  using A = typename Cplx<Real>::T;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x)
    psi[i] = ((i % dim) == hf) ? A{1, 0} : A{0, 0};
}

template <typename Real>
int launch_gates_t(void* psi, void* lam, const AdjPass& P, const AdjOp* d_ops, const double2* d_cs,
                   double* d_partials, bool dual, bool backward, int num_sms, cudaStream_t stream) {
  using A = typename Cplx<Real>::T;
  const size_t smem = sizeof(A) * ((size_t)(dual ? 2 : 1) << (P.L + P.H));
  auto launch = [&](auto kern) {
    // Every instantiation has the same pointer type, so the opt-in is set per
    // launch (an idempotent attribute write) rather than once per type.
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(2 * sizeof(A) << AdjCfg<Real>::TB));
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, AdjCfg<Real>::NT, smem);
    uint64_t grid = (uint64_t)num_sms * (per_sm < 1 ? 1 : per_sm);
    if (grid > P.num_tiles) grid = P.num_tiles;
    kern<<<(unsigned)grid, AdjCfg<Real>::NT, smem, stream>>>((A*)psi, (A*)lam, P, d_ops, d_cs, d_partials);
  };
  if (!dual) launch(k_adj_gates<Real, false, false>);
  else if (backward) launch(k_adj_gates<Real, true, true>);
  else launch(k_adj_gates<Real, true, false>);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

template <typename Real>
int launch_pauli_t(const void* psi, void* lam, const AdjPass& P, const AdjTerm* d_terms, bool accumulate,
                   bool energy, double* d_epart, int num_sms, cudaStream_t stream) {
  using A = typename Cplx<Real>::T;
  const size_t smem = sizeof(A) << (P.L + P.H);
  static bool set = false;
  if (!set) {
    cudaFuncSetAttribute(k_adj_pauli<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(sizeof(A) << AdjCfg<Real>::TB));
    set = true;
  }
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adj_pauli<Real>, AdjCfg<Real>::NT, smem);
  uint64_t grid = (uint64_t)num_sms * (per_sm < 1 ? 1 : per_sm);
  if (grid > P.num_tiles) grid = P.num_tiles;
  k_adj_pauli<Real><<<(unsigned)grid, AdjCfg<Real>::NT, smem, stream>>>((const A*)psi, (A*)lam, P, d_terms,
                                                                       accumulate ? 1 : 0, energy ? 1 : 0, d_epart);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

}  // namespace

int adj_tile_bits(int dtype, bool dual) {
  const int tb = dtype == MLB_C128 ? AdjCfg<double>::TB : AdjCfg<float>::TB;
  return dual ? tb : tb;  // both arrays share the CTA's shared memory at this size
}

int launch_adj_init(int dtype, void* psi, int n, uint64_t batch, uint64_t hf, cudaStream_t stream) {
  const uint64_t dim = 1ull << n, total = dim * batch;
  uint64_t grid = (total + 255) / 256;
  if (grid > 148ull * 32) grid = 148ull * 32;
  if (dtype == MLB_C128) k_adj_init<double><<<(unsigned)grid, 256, 0, stream>>>((double2*)psi, dim, total, hf);
  else k_adj_init<float><<<(unsigned)grid, 256, 0, stream>>>((float2*)psi, dim, total, hf);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

int launch_adj_gates(int dtype, void* psi, void* lam, const AdjPass& P, const AdjOp* d_ops, const double2* d_cs,
                     double* d_partials, bool dual, bool backward, int num_sms, cudaStream_t stream) {
  if (P.num_ops < 1 || P.num_ops > kMaxAdjOps || P.num_segments > kMaxAdjSegs || P.num_slots > kMaxAdjSlots)
    return MLB_ERR_INVALID_ARG;
  if (dtype == MLB_C128)
    return launch_gates_t<double>(psi, lam, P, d_ops, d_cs, d_partials, dual, backward, num_sms, stream);
  return launch_gates_t<float>(psi, lam, P, d_ops, d_cs, d_partials, dual, backward, num_sms, stream);
}

int launch_adj_pauli(int dtype, const void* psi, void* lam, const AdjPass& P, const AdjTerm* d_terms,
                     bool accumulate, bool energy, double* d_epart, int num_sms, cudaStream_t stream) {
  if (P.num_ops < 1 || P.num_ops > kMaxAdjTerms) return MLB_ERR_INVALID_ARG;
  if (dtype == MLB_C128)
    return launch_pauli_t<double>(psi, lam, P, d_terms, accumulate, energy, d_epart, num_sms, stream);
  return launch_pauli_t<float>(psi, lam, P, d_terms, accumulate, energy, d_epart, num_sms, stream);
}

int launch_adj_reduce(const double* d_partials, uint64_t tiles_per_state, int num_slots, uint64_t batch,
                      const int* d_param_of_slot, int num_params, double* d_out, cudaStream_t stream) {
  const uint64_t total = batch * (uint64_t)num_slots;
  uint64_t grid = (total + 127) / 128;
  if (grid < 1) grid = 1;
  if (grid > 148ull * 16) grid = 148ull * 16;
  k_adj_reduce<<<(unsigned)grid, 128, 0, stream>>>(d_partials, tiles_per_state, num_slots, batch, d_param_of_slot,
                                                   num_params, d_out);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

// ---------------------------------------------------------------------------
// Per-vector squared norms of a batch of complex64 states and the division
// of energies and gradients by them (the tensor-core forward sweep's norm
// drift cancels: E and dE/dtheta both carry |psi|^2).  One CTA per vector,
// a fixed-order tree: the result does not depend on scheduling.
// ---------------------------------------------------------------------------
namespace {
__global__ void __launch_bounds__(256) k_batch_norm(const float2* __restrict__ psi, uint64_t dim,
                                                    double* __restrict__ out) {
  __shared__ double red[256];
  const float2* v = psi + (uint64_t)blockIdx.x * dim;
  double acc = 0.0;
  for (uint64_t i = threadIdx.x; i < dim; i += 256) {
    const float2 a = v[i];
    acc += (double)a.x * a.x + (double)a.y * a.y;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// out = [B] energies, then [B][P] gradients
__global__ void k_divide_by_norm(double* __restrict__ out, uint64_t batch, int num_params,
                                 const double* __restrict__ nrm) {
  const uint64_t total = batch * (uint64_t)(1 + num_params);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = i < batch ? i : (i - batch) / (uint64_t)num_params;
    out[i] /= nrm[b];
  }
}
}  // namespace

int launch_batch_norm(const void* psi_c64, uint64_t dim, uint64_t batch, double* d_norm, cudaStream_t stream) {
  if (batch == 0 || batch > 65535) return MLB_ERR_INVALID_ARG;
  k_batch_norm<<<(unsigned)batch, 256, 0, stream>>>(static_cast<const float2*>(psi_c64), dim, d_norm);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

int launch_divide_by_norm(double* d_out, uint64_t batch, int num_params, const double* d_norm,
                          cudaStream_t stream) {
  const uint64_t total = batch * (uint64_t)(1 + num_params);
  uint64_t grid = (total + 255) / 256;
  if (grid < 1) grid = 1;
  if (grid > 148ull * 8) grid = 148ull * 8;
  k_divide_by_norm<<<(unsigned)grid, 256, 0, stream>>>(d_out, batch, num_params, d_norm);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

}  // namespace mlb
