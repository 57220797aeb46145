// forward_quad.cu -- the residual / stage / limiter kernels for quadrilaterals, p = 0..3.
#include "forward_dispatch.cuh"
#include "forward_launch.cuh"

namespace nzb {
namespace {

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

cudaError_t initial_launch_quad(const nzb_mesh& m, const nzb_physics& ph, const nzb_initial_args& a, cudaStream_t st) {
  const unsigned nb = (unsigned)((m.n_elem + 127) / 128);
  switch (m.order) {
    case 0: k_initial_state<1, 0, false><<<nb, 128, 0, st>>>(m, ph, a); break;
    case 1: k_initial_state<1, 1, false><<<nb, 128, 0, st>>>(m, ph, a); break;
    case 2: k_initial_state<1, 2, false><<<nb, 128, 0, st>>>(m, ph, a); break;
    case 3: k_initial_state<1, 3, false><<<nb, 128, 0, st>>>(m, ph, a); break;
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

cudaError_t prepare_split_quad(int order) {
  switch (order) {
    case 1: return prepare_split<1, 1, false>();
    case 2: return prepare_split<1, 2, false>();
    case 3: return prepare_split<1, 3, false>();
  }
  return cudaSuccess;
}

cudaError_t upload_tables_fwd_quad(const double* src, size_t count, size_t offset) {
  return cudaMemcpyToSymbol(c_tab, src, sizeof(double) * count, sizeof(double) * offset);
}

}  // namespace nzb
