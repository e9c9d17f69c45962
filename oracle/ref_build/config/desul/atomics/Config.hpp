/* Hand-written (oracle build): desul atomics for an OpenMP host build. */
#ifndef DESUL_ATOMICS_CONFIG_HPP_
#define DESUL_ATOMICS_CONFIG_HPP_
#define DESUL_ATOMICS_ENABLE_OPENMP
#endif
