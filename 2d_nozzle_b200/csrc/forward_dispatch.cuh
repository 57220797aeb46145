// forward_dispatch.cuh -- launchers of the forward (residual / stage / limiter)
// kernels, one translation unit per element kind (forward_tri.cu,
// forward_quad.cu) so they compile in parallel.  Each unit holds its own copy
// of the reference-element tables in constant memory.
#pragma once
#include <cuda_runtime.h>

#include "element.cuh"
#include "geometry.cuh"
#include "initial.cuh"
#include "observe.cuh"
#include "slope.cuh"

#ifndef NZB_INTERNAL
#define NZB_INTERNAL __attribute__((visibility("hidden")))
#endif

namespace nzb {

NZB_INTERNAL cudaError_t element_launch_tri(const nzb_mesh& m, const nzb_physics& ph, const Work& w, cudaStream_t st);
NZB_INTERNAL cudaError_t element_launch_quad(const nzb_mesh& m, const nzb_physics& ph, const Work& w, cudaStream_t st);
NZB_INTERNAL cudaError_t observables_launch_tri(const nzb_mesh& m, const nzb_physics& ph, const nzb_obs_args& a,
                                                cudaStream_t st);
NZB_INTERNAL cudaError_t observables_launch_quad(const nzb_mesh& m, const nzb_physics& ph, const nzb_obs_args& a,
                                                 cudaStream_t st);
NZB_INTERNAL cudaError_t geometry_launch_tri(const nzb_mesh& m, const nzb_geometry_args& a, cudaStream_t st);
NZB_INTERNAL cudaError_t geometry_launch_quad(const nzb_mesh& m, const nzb_geometry_args& a, cudaStream_t st);
NZB_INTERNAL cudaError_t gen_rate_launch(const nzb_gen_mesh& m, const nzb_physics& ph, int unfolded, const double* U,
                                         double* out, double* wave, double* fw, double* smax, cudaStream_t st);
NZB_INTERNAL cudaError_t gen_limit_launch(const nzb_gen_mesh& m, const nzb_physics& ph, double* U,
                                          unsigned long long* counters, cudaStream_t st);
NZB_INTERNAL cudaError_t gen_update_launch(const nzb_gen_mesh& m, const nzb_physics& ph, const nzb_gen_update_args& a,
                                           cudaStream_t st);
NZB_INTERNAL cudaError_t gen_superbee_launch(const nzb_gen_mesh& m, const nzb_physics& ph, double* U,
                                             const double* share, double* means, double* scale,
                                             unsigned long long* counters, cudaStream_t st);
NZB_INTERNAL cudaError_t gen_initial_launch(const nzb_gen_mesh& m, const nzb_physics& ph,
                                            const nzb_gen_initial_args& a, cudaStream_t st);
NZB_INTERNAL cudaError_t gen_observables_launch(const nzb_gen_mesh& m, const nzb_physics& ph,
                                                const nzb_gen_obs_args& a, cudaStream_t st);
NZB_INTERNAL cudaError_t gen_geometry_launch(const nzb_gen_mesh& m, const nzb_gen_geometry_args& a, cudaStream_t st);
NZB_INTERNAL cudaError_t initial_launch_tri(const nzb_mesh& m, const nzb_physics& ph, const nzb_initial_args& a,
                                            cudaStream_t st);
NZB_INTERNAL cudaError_t initial_launch_quad(const nzb_mesh& m, const nzb_physics& ph, const nzb_initial_args& a,
                                             cudaStream_t st);
// raise the split kernels' dynamic shared-memory limit for one order (current device)
NZB_INTERNAL cudaError_t prepare_split_tri(int order);
NZB_INTERNAL cudaError_t prepare_split_quad(int order);
NZB_INTERNAL cudaError_t upload_tables_fwd_tri(const double* src, size_t count, size_t offset);
NZB_INTERNAL cudaError_t upload_tables_fwd_quad(const double* src, size_t count, size_t offset);

}  // namespace nzb
