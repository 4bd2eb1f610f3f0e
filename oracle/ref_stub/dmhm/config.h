/* Hand-written build configuration for compiling the reference library as
   the CPU oracle (what the reference's CMake would generate with RELEASE on,
   underscore-suffixed BLAS/LAPACK symbols and MPI_IN_PLACE available). */
#pragma once
#ifndef DMHM_CONFIG_H
#define DMHM_CONFIG_H 1
#define DMHM_VERSION_MAJOR 0
#define DMHM_VERSION_MINOR 2
#define RELEASE
#define BLAS_POST
#define LAPACK_POST
#define HAVE_MPI_IN_PLACE
#define RESTRICT __restrict__
#endif
