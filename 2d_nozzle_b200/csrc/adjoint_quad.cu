// adjoint_quad.cu -- the adjoint kernels for quadrilaterals, p = 0..3.
#include "adjoint_dispatch.cuh"

namespace nzb {
namespace {

template <int K, int P, bool AFF>
cudaError_t launch_vjp(const nzb_mesh& m, const nzb_physics& ph, const AdjWork& w, cudaStream_t st) {
  if constexpr (P > 0) {
    if (m.vjp_split == SPLIT_T) {
      const unsigned nb = (unsigned)(m.vjp_blocks ? m.n_vjp_blocks : (m.n_elem + SPLIT_EB - 1) / SPLIT_EB);
      if (nb) k_vjp_split<K, P, AFF><<<nb, SPLIT_T * 32, VjpSplitSmem<K, P>::BYTES, st>>>(m, ph, w);
      return cudaGetLastError();
    }
  }
  const int64_t nb = m.vjp_blocks ? m.n_vjp_blocks : (m.n_elem + Launch<K, P>::NT - 1) / Launch<K, P>::NT;
  if (nb) k_vjp<K, P, AFF><<<(unsigned)nb, Launch<K, P>::NT, 0, st>>>(m, ph, w);
  return cudaGetLastError();
}

// The split kernel's dynamic shared memory can exceed the default 48 KB:
// raise each instantiation's limit (once per device, at table upload).
template <int K, int P, bool AFF>
cudaError_t prepare_vjp() {
  if constexpr (P == 0) {
    return cudaSuccess;
  } else {
    return cudaFuncSetAttribute(k_vjp_split<K, P, AFF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                VjpSplitSmem<K, P>::BYTES);
  }
}

template <int K, int P>
cudaError_t launch_coords(const nzb_mesh& m, const nzb_physics& ph, const CoordWork& w, cudaStream_t st) {
  k_vjp_coords<K, P><<<(unsigned)((m.n_elem + 127) / 128), 128, 0, st>>>(m, ph, w);
  return cudaGetLastError();
}

}  // namespace

cudaError_t vjp_launch_quad(const nzb_mesh& m, const nzb_physics& ph, const AdjWork& w, cudaStream_t st) {
  switch (m.order) {
    case 0: return launch_vjp<1, 0, false>(m, ph, w, st);
    case 1: return launch_vjp<1, 1, false>(m, ph, w, st);
    case 2: return launch_vjp<1, 2, false>(m, ph, w, st);
    case 3: return launch_vjp<1, 3, false>(m, ph, w, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t vjp_coords_launch_quad(const nzb_mesh& m, const nzb_physics& ph, const CoordWork& w, cudaStream_t st) {
  switch (m.order) {
    case 0: return launch_coords<1, 0>(m, ph, w, st);
    case 1: return launch_coords<1, 1>(m, ph, w, st);
    case 2: return launch_coords<1, 2>(m, ph, w, st);
    case 3: return launch_coords<1, 3>(m, ph, w, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t prepare_vjp_split_quad(int order) {
  switch (order) {
    case 0: return cudaSuccess;
    case 1: return prepare_vjp<1, 1, false>();
    case 2: return prepare_vjp<1, 2, false>();
    case 3: return prepare_vjp<1, 3, false>();
  }
  return cudaErrorInvalidValue;
}

cudaError_t upload_tables_quad(const double* src, size_t count, size_t offset) {
  return cudaMemcpyToSymbol(c_tab, src, sizeof(double) * count, sizeof(double) * offset);
}

}  // namespace nzb
