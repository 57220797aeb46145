// forward_quad.cu -- the residual / stage / limiter kernels for quadrilaterals, p = 0..3.
#include "forward_dispatch.cuh"

namespace nzb {
namespace {

// One residual, rate, stage or limiter pass: with the edge pass, k_edge first
// (the limiter alone needs no fluxes), then the element kernel.
// The Superbee limiter's three passes over the state V, written to out.
template <int K, int P, bool AFF>
cudaError_t superbee_passes(const nzb_mesh& m, const nzb_physics& ph, const double* V, double* out,
                            unsigned long long* counters, uint8_t* flags, cudaStream_t st) {
  const unsigned nb = (unsigned)((m.n_elem + 127) / 128);
  k_cell_means<K, P, AFF><<<nb, 128, 0, st>>>(m, V, m.lim_means);
  k_lim_scale<<<1, 1024, 0, st>>>(m.lim_means, m.n_elem, m.lim_scale);
  k_superbee<K, P, AFF><<<nb, 128, 0, st>>>(m, ph, V, out, counters, flags);
  return cudaGetLastError();
}

template <int K, int P, bool AFF>
cudaError_t launch(const nzb_mesh& m, const nzb_physics& ph, const Work& w, cudaStream_t st) {
  // Superbee (limiter 2): the element kernel leaves the stage unlimited, then three passes
  const bool sb = ph.limiter == 2 && P > 0 && (w.op == OP_STAGE || w.op == OP_LIMIT);
  if (sb && w.op == OP_LIMIT) return superbee_passes<K, P, AFF>(m, ph, w.V, w.out, w.counters, w.flags, st);
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
  if (sb) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return superbee_passes<K, P, AFF>(m, ph, w.out, w.out, w.counters, w.flags, st);
  }
  return cudaGetLastError();
}

template <int P>
void geometry(const nzb_mesh& m, const nzb_geometry_args& a, cudaStream_t st) {
  const unsigned ne = (unsigned)((m.n_elem + 127) / 128), nk = (unsigned)((m.n_edge + 127) / 128);
  k_elem_geometry<1, P, false><<<ne, 128, 0, st>>>(m, a);
  k_edge_geometry<1, P><<<nk, 128, 0, st>>>(m, a);
}

}  // namespace

cudaError_t element_launch_quad(const nzb_mesh& m, const nzb_physics& ph, const Work& w, cudaStream_t st) {
  switch (m.order) {
    case 0: return launch<1, 0, false>(m, ph, w, st);
    case 1: return launch<1, 1, false>(m, ph, w, st);
    case 2: return launch<1, 2, false>(m, ph, w, st);
    case 3: return launch<1, 3, false>(m, ph, w, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t observables_launch_quad(const nzb_mesh& m, const nzb_physics& ph, const nzb_obs_args& a, cudaStream_t st) {
  const unsigned nb = (unsigned)a.n_seg;
  switch (m.order) {
    case 0: k_observables<1, 0, false><<<nb, OBS_BT, 0, st>>>(m, ph, a); break;
    case 1: k_observables<1, 1, false><<<nb, OBS_BT, 0, st>>>(m, ph, a); break;
    case 2: k_observables<1, 2, false><<<nb, OBS_BT, 0, st>>>(m, ph, a); break;
    case 3: k_observables<1, 3, false><<<nb, OBS_BT, 0, st>>>(m, ph, a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t geometry_launch_quad(const nzb_mesh& m, const nzb_geometry_args& a, cudaStream_t st) {
  switch (m.order) {
    case 0: geometry<0>(m, a, st); break;
    case 1: geometry<1>(m, a, st); break;
    case 2: geometry<2>(m, a, st); break;
    case 3: geometry<3>(m, a, st); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t upload_tables_fwd_quad(const double* src, size_t count, size_t offset) {
  return cudaMemcpyToSymbol(c_tab, src, sizeof(double) * count, sizeof(double) * offset);
}

}  // namespace nzb
