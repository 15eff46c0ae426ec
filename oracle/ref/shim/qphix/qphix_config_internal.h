/* Configuration for compiling the reference's header-only code (geometry,
   BLAS, clover product, solvers) as a plain scalar CPU build.  Written for
   this harness; it replaces the header the reference's own build system
   would configure. */
#ifndef QPHIX_CONFIG_INTERNAL_H
#define QPHIX_CONFIG_INTERNAL_H
#define QPHIX_USE_MM_MALLOC
#define QPHIX_SCALAR
#define QPHIX_SCALAR_SOURCE
#define QPHIX_BUILD_CLOVER
#define QPHIX_BUILD_TWISTED_MASS
#define QPHIX_BUILD_TWISTED_MASS_WITH_CLOVER
#define QPHIX_LLC_CACHE_ALIGN 64
#endif
