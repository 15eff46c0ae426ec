/* Configuration for compiling the reference's header-only code (geometry,
   BLAS, clover product, solvers, and the Dslash classes over its generated
   kernels) as a CPU build.  Written for this harness; it replaces the header
   the reference's own build system would configure.  The scalar target is the
   default; QPHIX_REF_ISA_AVX512 selects the AVX-512 kernels. */
#ifndef QPHIX_CONFIG_INTERNAL_H
#define QPHIX_CONFIG_INTERNAL_H
#define QPHIX_USE_MM_MALLOC
#define QPHIX_SCALAR
#if defined(QPHIX_REF_ISA_AVX512)
#define QPHIX_AVX512_SOURCE
#else
#define QPHIX_SCALAR_SOURCE
#endif
#define QPHIX_BUILD_CLOVER
#define QPHIX_BUILD_TWISTED_MASS
#define QPHIX_BUILD_TWISTED_MASS_WITH_CLOVER
#define QPHIX_LLC_CACHE_ALIGN 64
#endif
