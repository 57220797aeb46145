// generic.cu -- launchers of the any-order / curved-element kernels (generic.cuh),
// instantiated per basis-size bucket.
#include "forward_dispatch.cuh"
#include "gen_geometry.cuh"
#include "gen_initial.cuh"
#include "gen_observe.cuh"
#include "generic.cuh"

namespace nzb {
namespace {

template <class F>
cudaError_t by_bucket(int np, F&& fn) {
  switch (gen_np_bucket(np)) {
    case 4: return fn(std::integral_constant<int, 4>{});
    case 6: return fn(std::integral_constant<int, 6>{});
    case 10: return fn(std::integral_constant<int, 10>{});
    case 16: return fn(std::integral_constant<int, 16>{});
    case 21: return fn(std::integral_constant<int, 21>{});
    case 28: return fn(std::integral_constant<int, 28>{});
    default: return fn(std::integral_constant<int, 36>{});
  }
}

unsigned blocks(int64_t n) { return (unsigned)((n + 127) / 128); }

}  // namespace

cudaError_t gen_rate_launch(const nzb_gen_mesh& m, const nzb_physics& ph, int unfolded, const double* U, double* out,
                            double* wave, double* fw, double* smax, cudaStream_t st) {
  k_gen_edge<<<blocks(m.n_int + m.n_bnd), 128, 0, st>>>(m, ph, U, fw, smax);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return by_bucket(m.np, [&](auto B) {
    k_gen_element<decltype(B)::value><<<blocks(m.n_elem), 128, 0, st>>>(m, ph, unfolded, U, fw, smax, out, wave);
    return cudaGetLastError();
  });
}

cudaError_t gen_limit_launch(const nzb_gen_mesh& m, const nzb_physics& ph, double* U, unsigned long long* counters,
                             cudaStream_t st) {
  return by_bucket(m.np, [&](auto B) {
    k_gen_limit<decltype(B)::value><<<blocks(m.n_elem), 128, 0, st>>>(m, ph, U, counters);
    return cudaGetLastError();
  });
}

cudaError_t gen_update_launch(const nzb_gen_mesh& m, const nzb_physics& ph, const nzb_gen_update_args& a,
                              cudaStream_t st) {
  k_gen_update<<<blocks(m.n_elem), 128, 0, st>>>(m, ph, a.stage, a.dt_factor, a.a, a.b, a.V, a.U0, a.F, a.wave, a.dt,
                                                  a.out, a.partial);
  return cudaGetLastError();
}

cudaError_t gen_superbee_launch(const nzb_gen_mesh& m, const nzb_physics& ph, double* U, const double* share,
                                double* means, double* scale, unsigned long long* counters, cudaStream_t st) {
  k_gen_cell_means<<<blocks(m.n_elem), 128, 0, st>>>(m, U, means);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_gen_lim_scale<<<1, 1024, 0, st>>>(means, m.n_elem, scale);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return by_bucket(m.np, [&](auto B) {
    k_gen_superbee<decltype(B)::value><<<blocks(m.n_elem), 128, 0, st>>>(m, ph, U, means, scale, share, counters);
    return cudaGetLastError();
  });
}

cudaError_t gen_initial_launch(const nzb_gen_mesh& m, const nzb_physics& ph, const nzb_gen_initial_args& a,
                               cudaStream_t st) {
  const int bytes = GenInitSmem{m.np, m.nqv, a.ng}.total() * (int)sizeof(double);
  k_gen_initial_state<<<(unsigned)m.n_elem, 128, bytes, st>>>(m, ph, a);
  return cudaGetLastError();
}

cudaError_t gen_observables_launch(const nzb_gen_mesh& m, const nzb_physics& ph, const nzb_gen_obs_args& a,
                                   cudaStream_t st) {
  k_gen_observables<<<1, OBS_BT, 0, st>>>(m, ph, a);
  return cudaGetLastError();
}

cudaError_t gen_geometry_launch(const nzb_gen_mesh& m, const nzb_gen_geometry_args& a, cudaStream_t st) {
  const int bytes = GenGeoSmem{m.np, m.nqv, a.ng}.total() * (int)sizeof(double);
  if (bytes > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(k_gen_elem_geometry, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
  }
  k_gen_elem_geometry<<<(unsigned)m.n_elem, 128, bytes, st>>>(m, a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (m.n_int + m.n_bnd > 0) k_gen_edge_geometry<<<blocks(m.n_int + m.n_bnd), 128, 0, st>>>(m, a);
  return cudaGetLastError();
}

}  // namespace nzb
