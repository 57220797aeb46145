// forward_launch.cuh -- the launch of one residual, rate, stage or limiter pass
// for one (kind, order, geometry layout), shared by forward_tri.cu and
// forward_quad.cu (each translation unit instantiates it for its own kind).
//
// Variants (nzb_mesh.split, nzb_mesh.edge_pass):
//   split = 4      k_split: four threads per element (split.cuh), p >= 1;
//   edge_pass = 1  k_edge (one thread per edge) then k_element with the
//                  fluxes lifted from the edge array;
//   otherwise      k_element: one thread per element, fluxes from both sides.
// With the Superbee limiter (limiter 2) the element kernel leaves the stage
// unlimited and three passes follow (cell means, their maximum -- per
// instance in a batch -- and the slope limiter with the positivity limiter).
#pragma once
#include <cuda_runtime.h>

#include "element.cuh"
#include "slope.cuh"
#include "split.cuh"

namespace nzb {
namespace {

template <int K, int P, bool AFF>
cudaError_t superbee_passes(const nzb_mesh& m, const nzb_physics& ph, const double* V, double* out,
                            unsigned long long* counters, uint8_t* flags, cudaStream_t st) {
  const unsigned nb = (unsigned)((m.n_elem + 127) / 128);
  k_cell_means<K, P, AFF><<<nb, 128, 0, st>>>(m, V, m.lim_means);
  if (m.elem_inst)
    k_lim_scale_inst<<<nb, 128, 0, st>>>(m.lim_means, m.n_elem, m.elem_inst, m.lim_scale);
  else
    k_lim_scale<<<1, 1024, 0, st>>>(m.lim_means, m.n_elem, m.lim_scale);
  k_superbee<K, P, AFF><<<nb, 128, 0, st>>>(m, ph, V, out, counters, flags);
  return cudaGetLastError();
}

template <int K, int P, bool AFF>
cudaError_t launch(const nzb_mesh& m, const nzb_physics& ph, const Work& w, cudaStream_t st) {
  const bool sb = ph.limiter == 2 && P > 0 && (w.op == OP_STAGE || w.op == OP_LIMIT);
  if (sb && w.op == OP_LIMIT) return superbee_passes<K, P, AFF>(m, ph, w.V, w.out, w.counters, w.flags, st);
  const bool lim = w.op == OP_STAGE || w.op == OP_LIMIT;
  bool done = false;
  if constexpr (P > 0) {
    if (m.split == SPLIT_T) {
      const unsigned nb = (unsigned)(m.fwd_blocks ? m.n_fwd_blocks : (m.n_elem + SPLIT_EB - 1) / SPLIT_EB);
      constexpr int SM = SplitSmem<K, P>::BYTES;
      if (nb == 0)
        ;  // an empty block list: nothing marches
      else if (lim)
        k_split<K, P, AFF, true><<<nb, SPLIT_T * 32, SM, st>>>(m, ph, w);
      else
        k_split<K, P, AFF, false><<<nb, SPLIT_T * 32, SM, st>>>(m, ph, w);
      done = true;
    }
  }
  if (!done) {
    constexpr int NT = Launch<K, P>::NT;
    const unsigned nb = (unsigned)(m.fwd_blocks ? m.n_fwd_blocks : (m.n_elem + NT - 1) / NT);
    const bool ep = m.edge_pass && w.op != OP_LIMIT;
    if (ep) {
      k_edge<K, P><<<(unsigned)((m.n_edge + 127) / 128), 128, 0, st>>>(m, ph, w.V);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return e;
    }
    if (nb == 0)
      ;  // an empty block list: nothing marches
    else if (lim && ep)
      k_element<K, P, AFF, true, true><<<nb, NT, 0, st>>>(m, ph, w);
    else if (lim)
      k_element<K, P, AFF, true, false><<<nb, NT, 0, st>>>(m, ph, w);
    else if (ep)
      k_element<K, P, AFF, false, true><<<nb, NT, 0, st>>>(m, ph, w);
    else
      k_element<K, P, AFF, false, false><<<nb, NT, 0, st>>>(m, ph, w);
  }
  if (sb) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return superbee_passes<K, P, AFF>(m, ph, w.out, w.out, w.counters, w.flags, st);
  }
  return cudaGetLastError();
}

// The split kernels' dynamic shared memory exceeds the default 48 KB limit at
// p = 3: raise each instantiation's limit (once per device, at table upload).
template <int K, int P, bool AFF>
cudaError_t prepare_split() {
  if constexpr (P == 0) {
    return cudaSuccess;
  } else {
    constexpr int SM = SplitSmem<K, P>::BYTES;
    cudaError_t e = cudaFuncSetAttribute(k_split<K, P, AFF, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_split<K, P, AFF, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SM);
    return e;
  }
}

}  // namespace
}  // namespace nzb
