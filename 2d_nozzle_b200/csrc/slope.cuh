// slope.cuh -- the Superbee TVB slope limiter (src/spatial/limiter.py:246-429).
//
// Per element and face: the element's own increment toward the face, d = its
// trace averaged over the face minus its cell average, against the jump of
// cell averages across the face, a = ubar(neighbour) - ubar; a face is quiet
// (factor 1) on a domain boundary, where |d| <= 1e-12, or where |d| is below
// the TVB threshold tvb * (A_e / A_domain) * max over the domain |ubar_s|;
// otherwise its factor is clip(superbee(a, d) / d, 0, 1) with superbee(a, b)
// = maxmod(minmod(2a, b), minmod(a, 2b)).  One factor per element, the
// minimum over faces and components, scales the whole element toward its
// cell average: U <- ubar + theta (U - ubar).  The positivity limiter follows,
// as apply_limiter does.  Three passes, since the threshold needs a maximum
// over the whole domain and the jumps need the neighbours' cell averages:
//   k_cell_means   ubar of every element;
//   k_lim_scale    max_e |ubar_s| per component (one block, order-free), or
//   k_lim_scale_inst  the same per instance of a batch (the maximum of the
//                  bit patterns of non-negative doubles, by atomics: exact and
//                  order-free);
//   k_superbee     the factor, the scaling and the positivity limiter.
// In a batch every instance is limited against its own domain (its own
// maximum and area shares, as its one-at-a-time solve would be), and the
// elements of retired instances are left untouched.
#pragma once
#include "element.cuh"

namespace nzb {

__device__ __forceinline__ double minmod(double a, double b) {
  return a * b <= 0.0 ? 0.0 : (fabs(a) < fabs(b) ? a : b);
}
__device__ __forceinline__ double maxmod(double a, double b) {
  return a * b <= 0.0 ? 0.0 : (fabs(a) > fabs(b) ? a : b);
}
__device__ __forceinline__ double superbee2(double a, double b) {
  return maxmod(minmod(2.0 * a, b), minmod(a, 2.0 * b));
}

template <int K, int P, bool AFF>
__global__ void __launch_bounds__(128) k_cell_means(const nzb_mesh m, const double* __restrict__ V,
                                                    double* __restrict__ means) {
  using S = Shape<K, P>;
  constexpr int NP = S::NP;
  const int64_t E = m.n_elem;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // a batch's per-instance maxima start from zero (k_lim_scale_inst follows on the same stream)
  if (m.elem_inst && blockIdx.x == 0)
    for (int k = threadIdx.x; k < 4 * m.n_inst; k += blockDim.x) m.lim_scale[k] = 0.0;
  if (e >= E) return;
  double mw[NP];
  mean_weights<K, P, AFF>(m, e, mw);
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < NP; ++i) acc = fma(mw[i], __ldg(V + (s * NP + i) * E + e), acc);
    means[s * E + e] = acc;
  }
}

// scale[s] = max_e |means[s, e]| (max is exact in any order).
static __global__ void __launch_bounds__(1024) k_lim_scale(const double* __restrict__ means, int64_t E,
                                                           double* __restrict__ scale) {
  __shared__ double red[4][32];
  double mx[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t e = threadIdx.x; e < E; e += blockDim.x)
#pragma unroll
    for (int s = 0; s < 4; ++s) mx[s] = fmax(mx[s], fabs(means[s * E + e]));
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    double v = mx[s];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[s][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v = fmax(v, red[threadIdx.x][k]);
    scale[threadIdx.x] = v;
  }
}

// scale[4 i + s] = max over instance i's elements of |means[s, e]|.  Values
// are non-negative, so their bit patterns order as the values do; NaN is
// dropped, as fmax drops it in k_lim_scale.  A warp whose elements all belong
// to one instance reduces first and issues one atomic per component.
static __global__ void __launch_bounds__(128) k_lim_scale_inst(const double* __restrict__ means, int64_t E,
                                                               const int32_t* __restrict__ elem_inst,
                                                               double* __restrict__ scale) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = e < E;
  const int inst = ok ? __ldg(elem_inst + e) : -1;
  const int inst0 = __shfl_sync(0xffffffffu, inst, 0);
  const bool uniform = __all_sync(0xffffffffu, ok && inst == inst0);
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    double v = ok ? fabs(means[s * E + e]) : 0.0;
    if (!(v == v)) v = 0.0;
    if (uniform) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
      if ((threadIdx.x & 31) == 0 && v > 0.0)
        atomicMax(reinterpret_cast<unsigned long long*>(scale + 4 * inst0 + s), (unsigned long long)__double_as_longlong(v));
    } else if (ok && v > 0.0) {
      atomicMax(reinterpret_cast<unsigned long long*>(scale + 4 * inst + s), (unsigned long long)__double_as_longlong(v));
    }
  }
}

// In place allowed (V may alias out): an element reads its own coefficients
// and only its neighbours' cell averages.
template <int K, int P, bool AFF>
__global__ void __launch_bounds__(128) k_superbee(const nzb_mesh m, const nzb_physics ph, const double* V,
                                                  double* out, unsigned long long* counters, uint8_t* flags) {
  using S = Shape<K, P>;
  constexpr int NP = S::NP, NQF = S::NQF, NF = S::NF, NE = S::NE;
  const int64_t E = m.n_elem;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int scaled = 0, repaired = 0;
  int inst = -1;
  if (e < E && m.elem_inst) inst = __ldg(m.elem_inst + e);
  if (e < E && (inst < 0 || __ldg(m.inst_status + inst) == 0)) {
    double u[NP][4], ub[4], sc[4];
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int s = 0; s < 4; ++s) u[i][s] = V[(s * NP + i) * E + e];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      ub[s] = __ldg(m.lim_means + s * E + e);
      sc[s] = __ldg(m.lim_scale + (inst < 0 ? 0 : 4 * inst) + s);
    }
    const double share = __ldg(m.elem_share + e);
    double wsum = 0.0;
#pragma unroll
    for (int q = 0; q < NQF; ++q) wsum += tab<K, P>(S::O_WF + q);
    double theta = 1.0;
    int sides = 0;
#pragma unroll
    for (int f = 0; f < NF; ++f) {  // unrolled: the edge nodes index registers at compile time
      const int code = __ldg(m.face_code + f * E + e);
      const int nb = __ldg(m.face_nbr + f * E + e);
      const int side = code & 1;
      sides |= side << f;
      if (nb < 0) continue;  // a boundary face is not limited against
      double tm[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int q = 0; q < NQF; ++q) {
        const double wq = tab<K, P>(S::O_WF + q);
        double tr[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int j = 0; j < NE; ++j) {
          const double c = pfe<K, P>(side, f, j, q);
          const int n = edge_node(K, P, f, j);
#pragma unroll
          for (int s = 0; s < 4; ++s) tr[s] = fma(c, u[n][s], tr[s]);
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) tm[s] = fma(wq, tr[s], tm[s]);
      }
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const double d = tm[s] / wsum - ub[s];
        const double a = __ldg(m.lim_means + s * E + nb) - ub[s];
        const bool quiet = fabs(d) <= 1e-12 || fabs(d) <= ph.tvb_constant * share * sc[s];
        if (!quiet) {
          double tf = superbee2(a, d) / d;
          tf = tf < 0.0 ? 0.0 : (tf > 1.0 ? 1.0 : tf);
          theta = tf < theta ? tf : theta;
        }
      }
    }
    bool changed = false;
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const double v = ub[s] + theta * (u[i][s] - ub[s]);
        changed |= v != u[i][s];
        u[i][s] = v;
      }
    limit_element<K, P, AFF>(RegCoef<NP>{u}, m, ph, e, sides, scaled, repaired);
    scaled |= changed ? 1 : 0;
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int s = 0; s < 4; ++s) out[(s * NP + i) * E + e] = u[i][s];
    if (flags) flags[e] = (uint8_t)(scaled | (repaired << 1));
  }
  if (counters) {
    const int ns = __syncthreads_count(scaled);
    const int nr = __syncthreads_count(repaired);
    if (threadIdx.x == 0) {
      if (ns) atomicAdd(counters + 0, (unsigned long long)ns);
      if (nr) atomicAdd(counters + 1, (unsigned long long)nr);
    }
  }
}

}  // namespace nzb
