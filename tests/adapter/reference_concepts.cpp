// Compile-only check of the drop-in boundary against the reference's own headers (test infrastructure):
//  * the library's C++ layer (terraneo_b200/cpp/tn) satisfies the reference's VectorLike, Block2VectorLike,
//    OperatorLike and SolverLike concepts (linalg/vector.hpp:8-52, linalg/operator.hpp:57-71,
//    linalg/solvers/solver.hpp:19-29), and the reference's own solver templates (PCG, FGMRES, Chebyshev,
//    power iteration) instantiate over the library's operators and vectors;
//  * the reference-side binding (terraneo_b200/cpp/reference/epsilon_divdiv_kerngen_b200.hpp) satisfies
//    OperatorLike on the reference's VectorQ1Vec and drives the reference's PCG.
#include <cmath>
#include <concepts>
#include <vector>

#include "linalg/vector_q1.hpp"
#include "linalg/operator.hpp"
#include "linalg/solvers/chebyshev.hpp"
#include "linalg/solvers/fgmres.hpp"
#include "linalg/solvers/pbicgstab.hpp"
#include "linalg/solvers/pcg.hpp"
#include "linalg/solvers/power_iteration.hpp"
#include "linalg/solvers/solver.hpp"
#include "linalg/vector.hpp"
#include "linalg/vector_q1.hpp"
#include "reference/epsilon_divdiv_kerngen_b200.hpp"
#include "tn/linalg.hpp"
#include "tn/operators.hpp"

namespace L = terra::linalg;
namespace S = terra::linalg::solvers;
using B200Op = terra::fe::wedge::operators::shell::EpsilonDivDivKerngenB200< double >;

static_assert( L::VectorLike< tn::VectorQ1Vec< double > > );
static_assert( L::VectorLike< tn::VectorQ1Vec< float > > );
static_assert( L::VectorLike< tn::VectorQ1Scalar< double > > );
static_assert( L::Block2VectorLike< tn::VectorQ1IsoQ2Q1< double > > );
static_assert( L::OperatorLike< tn::EpsilonDivDivKerngen< double > > );
static_assert( L::OperatorLike< tn::EpsilonDivDivKerngen< float > > );
static_assert( L::OperatorLike< tn::Laplace< double > > );
static_assert( L::OperatorLike< tn::EpsDivDivStokes< double > > );
static_assert( L::OperatorLike< tn::UnsteadyAdvectionDiffusionSUPG< double > > );
static_assert( L::OperatorLike< B200Op > );

// the reference's drivers over the library's operators and vectors
template class S::PCG< tn::EpsilonDivDivKerngen< double > >;
template class S::PCG< tn::Laplace< double > >;
template class S::Chebyshev< tn::EpsilonDivDivKerngen< double > >;
template class S::FGMRES< tn::EpsDivDivStokes< double > >;
template class S::PBiCGStab< tn::UnsteadyAdvectionDiffusionSUPG< double > >;
static_assert( S::SolverLike< S::PCG< tn::EpsilonDivDivKerngen< double > > > );
static_assert( S::SolverLike< S::Chebyshev< tn::EpsilonDivDivKerngen< double > > > );
static_assert( S::SolverLike< S::FGMRES< tn::EpsDivDivStokes< double > > > );
static_assert( S::SolverLike< S::PBiCGStab< tn::UnsteadyAdvectionDiffusionSUPG< double > > > );
template double S::power_iteration< tn::EpsilonDivDivKerngen< double > >( tn::EpsilonDivDivKerngen< double >&,
                                                                           tn::VectorQ1Vec< double >&,
                                                                           tn::VectorQ1Vec< double >&, int );

// ... and over the reference-side binding on the reference's own vectors
template class S::PCG< B200Op >;
static_assert( S::SolverLike< S::PCG< B200Op > > );

int main() { return 0; }
