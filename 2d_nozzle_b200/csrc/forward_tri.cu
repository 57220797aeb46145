// forward_tri.cu -- the residual / stage / limiter kernels for triangles, p = 0..3.
#include "forward_dispatch.cuh"

namespace nzb {
namespace {

// One residual, rate, stage or limiter pass: with the edge pass, k_edge first
// (the limiter alone needs no fluxes), then the element kernel.
template <int K, int P, bool AFF>
cudaError_t launch(const nzb_mesh& m, const nzb_physics& ph, const Work& w, cudaStream_t st) {
  constexpr int NT = Launch<K, P>::NT;
  const unsigned nb = (unsigned)((m.n_elem + NT - 1) / NT);
  const bool lim = w.op == OP_STAGE || w.op == OP_LIMIT;
  const bool ep = m.edge_pass && w.op != OP_LIMIT;
  if (ep) {
    k_edge<K, P><<<(unsigned)((m.n_edge + 127) / 128), 128, 0, st>>>(m, ph, w.V);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (lim && ep)
    k_element<K, P, AFF, true, true><<<nb, NT, 0, st>>>(m, ph, w);
  else if (lim)
    k_element<K, P, AFF, true, false><<<nb, NT, 0, st>>>(m, ph, w);
  else if (ep)
    k_element<K, P, AFF, false, true><<<nb, NT, 0, st>>>(m, ph, w);
  else
    k_element<K, P, AFF, false, false><<<nb, NT, 0, st>>>(m, ph, w);
  return cudaGetLastError();
}

}  // namespace

cudaError_t element_launch_tri(const nzb_mesh& m, const nzb_physics& ph, const Work& w, cudaStream_t st) {
  switch (m.order) {
    case 0: return m.affine ? launch<0, 0, true>(m, ph, w, st) : launch<0, 0, false>(m, ph, w, st);
    case 1: return m.affine ? launch<0, 1, true>(m, ph, w, st) : launch<0, 1, false>(m, ph, w, st);
    case 2: return m.affine ? launch<0, 2, true>(m, ph, w, st) : launch<0, 2, false>(m, ph, w, st);
    case 3: return m.affine ? launch<0, 3, true>(m, ph, w, st) : launch<0, 3, false>(m, ph, w, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t upload_tables_fwd_tri(const double* src, size_t count, size_t offset) {
  return cudaMemcpyToSymbol(c_tab, src, sizeof(double) * count, sizeof(double) * offset);
}

}  // namespace nzb
