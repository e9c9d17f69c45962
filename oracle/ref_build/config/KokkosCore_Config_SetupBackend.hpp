/* Hand-written (oracle build): host backends need no setup header. */
#ifndef KOKKOS_SETUP_HPP_
#define KOKKOS_SETUP_HPP_
#endif
