/* Hand-written Kokkos 4.6.01 configuration for the oracle build of the
 * reference (host only: OpenMP default execution space + Serial).
 * Equivalent to configuring the vendored Kokkos with
 *   -DKokkos_ENABLE_OPENMP=ON -DKokkos_ENABLE_SERIAL=ON -DCMAKE_CXX_STANDARD=20
 * This file is test infrastructure: it lets oracle/ref_build/Makefile compile
 * the reference with g++ directly, without the reference's cmake build. */
#if !defined(KOKKOS_MACROS_HPP) || defined(KOKKOS_CORE_CONFIG_H)
#error "Do not include KokkosCore_config.h directly; include Kokkos_Macros.hpp instead."
#else
#define KOKKOS_CORE_CONFIG_H
#endif
#define KOKKOS_VERSION 40601
#define KOKKOS_VERSION_MAJOR 4
#define KOKKOS_VERSION_MINOR 6
#define KOKKOS_VERSION_PATCH 1
#define KOKKOS_ENABLE_SERIAL
#define KOKKOS_ENABLE_OPENMP
#define KOKKOS_ENABLE_CXX20
#define KOKKOS_ENABLE_DEPRECATED_CODE_4
#define KOKKOS_ENABLE_COMPLEX_ALIGN
#define KOKKOS_ENABLE_LIBDL
