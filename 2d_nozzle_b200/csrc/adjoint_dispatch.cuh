// adjoint_dispatch.cuh -- launchers of the adjoint kernels, one translation unit
// per element kind (adjoint_tri.cu, adjoint_quad.cu) so the dual-number kernels
// compile in parallel.  Each unit holds its own copy of the reference-element
// tables in constant memory; nzb_upload_tables fills every copy.
#pragma once
#include <cuda_runtime.h>

#include "adjoint.cuh"
#include "adjoint_split.cuh"

#ifndef NZB_INTERNAL
#define NZB_INTERNAL __attribute__((visibility("hidden")))
#endif

namespace nzb {

NZB_INTERNAL cudaError_t vjp_launch_tri(const nzb_mesh& m, const nzb_physics& ph, const AdjWork& w, cudaStream_t st);
NZB_INTERNAL cudaError_t vjp_launch_quad(const nzb_mesh& m, const nzb_physics& ph, const AdjWork& w, cudaStream_t st);
NZB_INTERNAL cudaError_t vjp_coords_launch_tri(const nzb_mesh& m, const nzb_physics& ph, const CoordWork& w,
                                               cudaStream_t st);
NZB_INTERNAL cudaError_t vjp_coords_launch_quad(const nzb_mesh& m, const nzb_physics& ph, const CoordWork& w,
                                                cudaStream_t st);
NZB_INTERNAL cudaError_t prepare_vjp_split_tri(int order);
NZB_INTERNAL cudaError_t prepare_vjp_split_quad(int order);
NZB_INTERNAL cudaError_t upload_tables_tri(const double* src, size_t count, size_t offset);
NZB_INTERNAL cudaError_t upload_tables_quad(const double* src, size_t count, size_t offset);

}  // namespace nzb
