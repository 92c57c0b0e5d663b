// Stand-in for the configuration header that the reference's CMake build
// generates from include/ginkgo/config.hpp.in.  It lets the maintainer-side
// shim (tests/shim/ginkgo_b200_cuda_shim.cpp) be compiled against the
// reference's headers as a signature check, without running the reference's
// build system.  Values: version 1.12.0, mixed precision on, no optional
// third-party libraries.
#ifndef GKO_INCLUDE_CONFIG_H
#define GKO_INCLUDE_CONFIG_H

#define GKO_VERSION_MAJOR 1
#define GKO_VERSION_MINOR 12
#define GKO_VERSION_PATCH 0
#define GKO_VERSION_TAG "main"
#define GKO_VERSION_STR 1, 12, 0
#define GINKGO_VERSION_TAG_DEPRECATED 0
#define GKO_VERBOSE_LEVEL 1
#define GKO_HAVE_CXXABI_H
#define GKO_SIZE_T_IS_UINT64_T
#define GINKGO_MIXED_PRECISION
#define GINKGO_HIP_PLATFORM_HCC 0
#define GINKGO_HIP_PLATFORM_NVCC 0
#define GINKGO_DPCPP_MAJOR_VERSION 0
#define GINKGO_DPCPP_MINOR_VERSION 0
#define GKO_HAVE_PAPI_SDE 0
#define GKO_HAVE_TAU 0
#define GKO_HAVE_VTUNE 0
#define GKO_HAVE_METIS 0
#define GKO_HAVE_ROCTX 0
#define GINKGO_BUILD_MPI 0
#define GINKGO_HAVE_GPU_AWARE_MPI 0
#define GKO_HAVE_HWLOC 0
#define GINKGO_ENABLE_HALF 1
#define GINKGO_ENABLE_BFLOAT16 1
#define GINKGO_HAVE_OPENMPI_PRE_4_1_X 0

#endif  // GKO_INCLUDE_CONFIG_H
