// forward_tri.cu -- the residual / stage / limiter kernels for triangles, p = 0..3.
#include "forward_dispatch.cuh"
#include "forward_launch.cuh"

namespace nzb {
namespace {

template <int P>
void observe(const nzb_mesh& m, const nzb_physics& ph, const nzb_obs_args& a, cudaStream_t st) {
  if (m.affine)
    k_observables<0, P, true><<<(unsigned)a.n_seg, OBS_BT, 0, st>>>(m, ph, a);
  else
    k_observables<0, P, false><<<(unsigned)a.n_seg, OBS_BT, 0, st>>>(m, ph, a);
}

template <int P>
void geometry(const nzb_mesh& m, const nzb_geometry_args& a, cudaStream_t st) {
  const unsigned ne = (unsigned)((m.n_elem + 127) / 128), nk = (unsigned)((m.n_edge + 127) / 128);
  if (m.affine)
    k_elem_geometry<0, P, true><<<ne, 128, 0, st>>>(m, a);
  else
    k_elem_geometry<0, P, false><<<ne, 128, 0, st>>>(m, a);
  k_edge_geometry<0, P><<<nk, 128, 0, st>>>(m, a);
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

cudaError_t observables_launch_tri(const nzb_mesh& m, const nzb_physics& ph, const nzb_obs_args& a, cudaStream_t st) {
  switch (m.order) {
    case 0: observe<0>(m, ph, a, st); break;
    case 1: observe<1>(m, ph, a, st); break;
    case 2: observe<2>(m, ph, a, st); break;
    case 3: observe<3>(m, ph, a, st); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t initial_launch_tri(const nzb_mesh& m, const nzb_physics& ph, const nzb_initial_args& a, cudaStream_t st) {
  const unsigned nb = (unsigned)((m.n_elem + 127) / 128);
  switch (m.order * 2 + (m.affine ? 1 : 0)) {
    case 0: k_initial_state<0, 0, false><<<nb, 128, 0, st>>>(m, ph, a); break;
    case 1: k_initial_state<0, 0, true><<<nb, 128, 0, st>>>(m, ph, a); break;
    case 2: k_initial_state<0, 1, false><<<nb, 128, 0, st>>>(m, ph, a); break;
    case 3: k_initial_state<0, 1, true><<<nb, 128, 0, st>>>(m, ph, a); break;
    case 4: k_initial_state<0, 2, false><<<nb, 128, 0, st>>>(m, ph, a); break;
    case 5: k_initial_state<0, 2, true><<<nb, 128, 0, st>>>(m, ph, a); break;
    case 6: k_initial_state<0, 3, false><<<nb, 128, 0, st>>>(m, ph, a); break;
    case 7: k_initial_state<0, 3, true><<<nb, 128, 0, st>>>(m, ph, a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t geometry_launch_tri(const nzb_mesh& m, const nzb_geometry_args& a, cudaStream_t st) {
  switch (m.order) {
    case 0: geometry<0>(m, a, st); break;
    case 1: geometry<1>(m, a, st); break;
    case 2: geometry<2>(m, a, st); break;
    case 3: geometry<3>(m, a, st); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t prepare_split_tri(int order) {
  switch (order) {
    case 1: {
      const cudaError_t e = prepare_split<0, 1, true>();
      return e != cudaSuccess ? e : prepare_split<0, 1, false>();
    }
    case 2: {
      const cudaError_t e = prepare_split<0, 2, true>();
      return e != cudaSuccess ? e : prepare_split<0, 2, false>();
    }
    case 3: {
      const cudaError_t e = prepare_split<0, 3, true>();
      return e != cudaSuccess ? e : prepare_split<0, 3, false>();
    }
  }
  return cudaSuccess;
}

cudaError_t upload_tables_fwd_tri(const double* src, size_t count, size_t offset) {
  return cudaMemcpyToSymbol(c_tab, src, sizeof(double) * count, sizeof(double) * offset);
}

}  // namespace nzb
