// C++ mirror of the reference's operator concept (linalg/operator.hpp:57-71)
// over the terraneo_b200 C ABI: apply_impl(src, dst), apply / communication
// modes, diagonal mode and boundary conditions, with the reference's class
// names (fe/wedge/operators/shell/*.hpp).
#pragma once

#include "linalg.hpp"

namespace tn {

enum class OperatorApplyMode
{
    Replace = TN_APPLY_REPLACE,
    Add     = TN_APPLY_ADD
};
enum class OperatorCommunicationMode
{
    SkipCommunication     = TN_COMM_SKIP,
    CommunicateAdditively = TN_COMM_ADDITIVE
};

struct BoundaryConditions
{
    int cmb = TN_BC_DIRICHLET, surface = TN_BC_DIRICHLET;
};

// EpsilonDivDivKerngen (epsilon_divdiv_kerngen.hpp:62)
template < typename T >
class EpsilonDivDivKerngen
{
  public:
    using SrcVectorType = VectorQ1Vec< T >;
    using DstVectorType = VectorQ1Vec< T >;
    using ScalarType    = T;

    EpsilonDivDivKerngen() = default;
    EpsilonDivDivKerngen( const Mesh& mesh, const VectorQ1Scalar< T >& k, BoundaryConditions bcs, bool diagonal,
                          OperatorApplyMode         am = OperatorApplyMode::Replace,
                          OperatorCommunicationMode cm = OperatorCommunicationMode::CommunicateAdditively )
    : mesh_( mesh )
    , k_( k )
    {
        p_ = tn_epsdivdiv_params{ bcs.cmb, bcs.surface, diagonal ? 1 : 0, int( am ), int( cm ), 1.0 };
    }
    void set_operator_apply_and_communication_modes( OperatorApplyMode am, OperatorCommunicationMode cm )
    {
        p_.apply_mode = int( am ), p_.comm_mode = int( cm );
    }
    void set_diagonal( bool v ) { p_.diagonal = v ? 1 : 0; }
    void set_penalty_epsilon( double e ) { p_.penalty_eps = e; }
    void set_boundary_conditions( BoundaryConditions b ) { p_.bc_cmb = b.cmb, p_.bc_surface = b.surface; }
    const Mesh& get_domain() const { return mesh_; }
    const VectorQ1Scalar< T >& k_grid_data() const { return k_; }

    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        const T* s[3] = { src.comp( 0 ), src.comp( 1 ), src.comp( 2 ) };
        T*       d[3];
        dst.ptrs( d );
        if constexpr ( std::is_same_v< T, double > )
            check( tn_epsdivdiv_apply_f64( mesh_.get(), &p_, k_.comp( 0 ), s, d, stream() ), "epsdivdiv apply" );
        else
            check( tn_epsdivdiv_apply_f32( mesh_.get(), &p_, k_.comp( 0 ), s, d, stream() ), "epsdivdiv apply" );
    }

  private:
    Mesh                mesh_;
    VectorQ1Scalar< T > k_;
    tn_epsdivdiv_params p_{};
};

// EpsilonDivDivKerngen with OperatorStoredMatrixMode::Full: stored 18x18
// wedge matrices (tn_stored_epsdivdiv_apply_*), e.g. GCA coarse operators
template < typename T >
class StoredEpsilonDivDiv
{
  public:
    using SrcVectorType = VectorQ1Vec< T >;
    using DstVectorType = VectorQ1Vec< T >;
    using ScalarType    = T;
    StoredEpsilonDivDiv() = default;
    StoredEpsilonDivDiv( const Mesh& mesh, std::shared_ptr< T > mats, BoundaryConditions bcs, bool diagonal = false )
    : mesh_( mesh ), mats_( std::move( mats ) )
    {
        p_ = tn_epsdivdiv_params{ bcs.cmb, bcs.surface, diagonal ? 1 : 0, TN_APPLY_REPLACE, TN_COMM_ADDITIVE, 1.0 };
    }
    void set_operator_apply_and_communication_modes( OperatorApplyMode am, OperatorCommunicationMode cm )
    {
        p_.apply_mode = int( am ), p_.comm_mode = int( cm );
    }
    void set_diagonal( bool v ) { p_.diagonal = v ? 1 : 0; }
    const Mesh&                mesh() const { return mesh_; }
    const T*                   matrices() const { return mats_.get(); }
    const tn_epsdivdiv_params& params() const { return p_; }
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        const T* s[3] = { src.comp( 0 ), src.comp( 1 ), src.comp( 2 ) };
        T*       d[3];
        dst.ptrs( d );
        if constexpr ( std::is_same_v< T, double > )
            check( tn_stored_epsdivdiv_apply_f64( mesh_.get(), mats_.get(), &p_, s, d, stream() ), "stored apply" );
        else
            check( tn_stored_epsdivdiv_apply_f32( mesh_.get(), mats_.get(), &p_, s, d, stream() ), "stored apply" );
    }

  private:
    Mesh                 mesh_;
    std::shared_ptr< T > mats_;
    tn_epsdivdiv_params  p_{};
};

// The viscous operator of one multigrid level: matrix-free kerngen or stored
// matrices, chosen at run time (copies share the underlying operator)
template < typename T >
class ViscousOp
{
  public:
    using SrcVectorType = VectorQ1Vec< T >;
    using DstVectorType = VectorQ1Vec< T >;
    using ScalarType    = T;
    ViscousOp() = default;
    explicit ViscousOp( std::shared_ptr< EpsilonDivDivKerngen< T > > k ) : k_( std::move( k ) ) {}
    explicit ViscousOp( std::shared_ptr< StoredEpsilonDivDiv< T > > s ) : s_( std::move( s ) ) {}
    void set_diagonal( bool v )
    {
        if ( k_ )
            k_->set_diagonal( v );
        else
            s_->set_diagonal( v );
    }
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        if ( k_ )
            k_->apply_impl( src, dst );
        else
            s_->apply_impl( src, dst );
    }
    // the stored-matrix operator, or nullptr for the matrix-free one
    const StoredEpsilonDivDiv< T >* stored() const { return s_.get(); }

  private:
    std::shared_ptr< EpsilonDivDivKerngen< T > > k_;
    std::shared_ptr< StoredEpsilonDivDiv< T > >  s_;
};

// Laplace (laplace.hpp:18)
template < typename T >
class Laplace
{
  public:
    using SrcVectorType = VectorQ1Scalar< T >;
    using DstVectorType = VectorQ1Scalar< T >;
    using ScalarType    = T;
    Laplace( const Mesh& mesh, bool treat_boundary, bool diagonal ) : mesh_( mesh ), treat_( treat_boundary ), diag_( diagonal ) {}
    void set_operator_apply_and_communication_modes( OperatorApplyMode am, OperatorCommunicationMode cm )
    {
        am_ = am, cm_ = cm;
    }
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        if constexpr ( std::is_same_v< T, double > )
            check( tn_laplace_apply_f64( mesh_.get(), treat_, diag_, int( am_ ), int( cm_ ), src.comp( 0 ), dst.comp( 0 ),
                                         stream() ),
                   "laplace apply" );
        else
            check( tn_laplace_apply_f32( mesh_.get(), treat_, diag_, int( am_ ), int( cm_ ), src.comp( 0 ), dst.comp( 0 ),
                                         stream() ),
                   "laplace apply" );
    }

  private:
    Mesh                      mesh_;
    bool                      treat_, diag_;
    OperatorApplyMode         am_ = OperatorApplyMode::Replace;
    OperatorCommunicationMode cm_ = OperatorCommunicationMode::CommunicateAdditively;
};

// DivKGrad (div_k_grad.hpp:18): int k grad u . grad v
template < typename T >
class DivKGrad
{
  public:
    using SrcVectorType = VectorQ1Scalar< T >;
    using DstVectorType = VectorQ1Scalar< T >;
    using ScalarType    = T;
    DivKGrad( const Mesh& mesh, const VectorQ1Scalar< T >& k, bool treat_boundary, bool diagonal = false )
    : mesh_( mesh ), k_( k ), treat_( treat_boundary ), diag_( diagonal )
    {}
    void set_diagonal( bool v ) { diag_ = v; }
    void set_single_quadpoint( bool v ) { single_ = v; }
    void set_operator_apply_and_communication_modes( OperatorApplyMode am, OperatorCommunicationMode cm )
    {
        am_ = am, cm_ = cm;
    }
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        if constexpr ( std::is_same_v< T, double > )
            check( tn_divkgrad_apply_f64( mesh_.get(), k_.comp( 0 ), treat_, diag_, single_, int( am_ ), int( cm_ ),
                                          src.comp( 0 ), dst.comp( 0 ), stream() ),
                   "divkgrad apply" );
        else
            check( tn_divkgrad_apply_f32( mesh_.get(), k_.comp( 0 ), treat_, diag_, single_, int( am_ ), int( cm_ ),
                                          src.comp( 0 ), dst.comp( 0 ), stream() ),
                   "divkgrad apply" );
    }

  private:
    Mesh                      mesh_;
    VectorQ1Scalar< T >       k_;
    bool                      treat_, diag_, single_ = false;
    OperatorApplyMode         am_ = OperatorApplyMode::Replace;
    OperatorCommunicationMode cm_ = OperatorCommunicationMode::CommunicateAdditively;
};

// Gradient (gradient.hpp:28): coarse pressure -> fine velocity
template < typename T >
class Gradient
{
  public:
    using SrcVectorType = VectorQ1Scalar< T >;
    using DstVectorType = VectorQ1Vec< T >;
    using ScalarType    = T;
    Gradient() = default;
    Gradient( const Mesh& mu, const Mesh& mp, BoundaryConditions bcs ) : mu_( mu ), mp_( mp ), bcs_( bcs ) {}
    void set_operator_apply_and_communication_modes( OperatorApplyMode am, OperatorCommunicationMode cm )
    {
        am_ = am, cm_ = cm;
    }
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        T* d[3];
        dst.ptrs( d );
        if constexpr ( std::is_same_v< T, double > )
            check( tn_gradient_apply_f64( mu_.get(), mp_.get(), bcs_.cmb, bcs_.surface, int( am_ ), int( cm_ ),
                                          src.comp( 0 ), d, stream() ),
                   "gradient apply" );
        else
            check( tn_gradient_apply_f32( mu_.get(), mp_.get(), bcs_.cmb, bcs_.surface, int( am_ ), int( cm_ ),
                                          src.comp( 0 ), d, stream() ),
                   "gradient apply" );
    }

  private:
    Mesh                      mu_, mp_;
    BoundaryConditions        bcs_;
    OperatorApplyMode         am_ = OperatorApplyMode::Replace;
    OperatorCommunicationMode cm_ = OperatorCommunicationMode::CommunicateAdditively;
};

// Divergence (divergence.hpp:30): fine velocity -> coarse pressure
template < typename T >
class Divergence
{
  public:
    using SrcVectorType = VectorQ1Vec< T >;
    using DstVectorType = VectorQ1Scalar< T >;
    using ScalarType    = T;
    Divergence() = default;
    Divergence( const Mesh& mu, const Mesh& mp, BoundaryConditions bcs ) : mu_( mu ), mp_( mp ), bcs_( bcs ) {}
    void set_operator_apply_and_communication_modes( OperatorApplyMode am, OperatorCommunicationMode cm )
    {
        am_ = am, cm_ = cm;
    }
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        const T* s[3] = { src.comp( 0 ), src.comp( 1 ), src.comp( 2 ) };
        if constexpr ( std::is_same_v< T, double > )
            check( tn_divergence_apply_f64( mu_.get(), mp_.get(), bcs_.cmb, bcs_.surface, int( am_ ), int( cm_ ), s,
                                            dst.comp( 0 ), stream() ),
                   "divergence apply" );
        else
            check( tn_divergence_apply_f32( mu_.get(), mp_.get(), bcs_.cmb, bcs_.surface, int( am_ ), int( cm_ ), s,
                                            dst.comp( 0 ), stream() ),
                   "divergence apply" );
    }

  private:
    Mesh                      mu_, mp_;
    BoundaryConditions        bcs_;
    OperatorApplyMode         am_ = OperatorApplyMode::Replace;
    OperatorCommunicationMode cm_ = OperatorCommunicationMode::CommunicateAdditively;
};

// EpsDivDivStokes (epsilon_divdiv_stokes.hpp:19): [A B^T; B 0]
template < typename T >
class EpsDivDivStokes
{
  public:
    using SrcVectorType = VectorQ1IsoQ2Q1< T >;
    using DstVectorType = VectorQ1IsoQ2Q1< T >;
    using ScalarType    = T;
    using Block11Type   = EpsilonDivDivKerngen< T >;
    using Block12Type   = Gradient< T >;
    using Block21Type   = Divergence< T >;

    EpsDivDivStokes( const Mesh& mu, const Mesh& mp, const VectorQ1Scalar< T >& k, BoundaryConditions bcs )
    : A_( mu, k, bcs, false )
    , BT_( mu, mp, bcs )
    , B_( mu, mp, bcs )
    {}
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        // A (Replace, no halo) + B^T (Add, halo): one velocity halo per Stokes apply (:55-90)
        A_.set_operator_apply_and_communication_modes( OperatorApplyMode::Replace,
                                                       OperatorCommunicationMode::SkipCommunication );
        BT_.set_operator_apply_and_communication_modes( OperatorApplyMode::Add,
                                                        OperatorCommunicationMode::CommunicateAdditively );
        B_.set_operator_apply_and_communication_modes( OperatorApplyMode::Replace,
                                                       OperatorCommunicationMode::CommunicateAdditively );
        apply( A_, src.block_1(), dst.block_1() );
        apply( BT_, src.block_2(), dst.block_1() );
        apply( B_, src.block_1(), dst.block_2() );
        A_.set_operator_apply_and_communication_modes( OperatorApplyMode::Replace,
                                                       OperatorCommunicationMode::CommunicateAdditively );
        BT_.set_operator_apply_and_communication_modes( OperatorApplyMode::Replace,
                                                        OperatorCommunicationMode::CommunicateAdditively );
    }
    Block11Type& block_11() { return A_; }
    Block12Type& block_12() { return BT_; }
    Block21Type& block_21() { return B_; }

  private:
    Block11Type A_;
    Block12Type BT_;
    Block21Type B_;
};

// constant transfers (prolongation_constant.hpp:103, restriction_constant.hpp:134)
template < typename T >
class ProlongationVecConstant
{
  public:
    using SrcVectorType = VectorQ1Vec< T >;
    using DstVectorType = VectorQ1Vec< T >;
    ProlongationVecConstant( const Mesh& fine, const Mesh& coarse, OperatorApplyMode am = OperatorApplyMode::Replace )
    : f_( fine ), c_( coarse ), am_( am )
    {}
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        const T* s[3] = { src.comp( 0 ), src.comp( 1 ), src.comp( 2 ) };
        T*       d[3];
        dst.ptrs( d );
        if constexpr ( std::is_same_v< T, double > )
            check( tn_prolongation_constant_f64( f_.get(), c_.get(), 3, int( am_ ), s, d, stream() ), "prolongation" );
        else
            check( tn_prolongation_constant_f32( f_.get(), c_.get(), 3, int( am_ ), s, d, stream() ), "prolongation" );
    }

  private:
    Mesh              f_, c_;
    OperatorApplyMode am_;
};

// ProlongationLinear / RestrictionLinear (prolongation_linear.hpp:15,
// restriction_linear.hpp:15) on scalar fields
template < typename T >
class ProlongationLinear
{
  public:
    using SrcVectorType = VectorQ1Scalar< T >;
    using DstVectorType = VectorQ1Scalar< T >;
    ProlongationLinear( const Mesh& fine, const Mesh& coarse, OperatorApplyMode am = OperatorApplyMode::Replace )
    : f_( fine ), c_( coarse ), am_( am )
    {}
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        const T* s[1] = { src.comp( 0 ) };
        T*       d[1] = { dst.comp( 0 ) };
        if constexpr ( std::is_same_v< T, double > )
            check( tn_prolongation_linear_f64( f_.get(), c_.get(), 1, int( am_ ), s, d, stream() ), "prolongation" );
        else
            check( tn_prolongation_linear_f32( f_.get(), c_.get(), 1, int( am_ ), s, d, stream() ), "prolongation" );
    }

  private:
    Mesh              f_, c_;
    OperatorApplyMode am_;
};

template < typename T >
class RestrictionLinear
{
  public:
    using SrcVectorType = VectorQ1Scalar< T >;
    using DstVectorType = VectorQ1Scalar< T >;
    RestrictionLinear( const Mesh& fine, const Mesh& coarse ) : f_( fine ), c_( coarse ) {}
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        const T* s[1] = { src.comp( 0 ) };
        T*       d[1] = { dst.comp( 0 ) };
        if constexpr ( std::is_same_v< T, double > )
            check( tn_restriction_linear_f64( f_.get(), c_.get(), 1, s, d, stream() ), "restriction" );
        else
            check( tn_restriction_linear_f32( f_.get(), c_.get(), 1, s, d, stream() ), "restriction" );
    }

  private:
    Mesh f_, c_;
};

template < typename T >
class RestrictionVecConstant
{
  public:
    using SrcVectorType = VectorQ1Vec< T >;
    using DstVectorType = VectorQ1Vec< T >;
    RestrictionVecConstant( const Mesh& fine, const Mesh& coarse ) : f_( fine ), c_( coarse ) {}
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        const T* s[3] = { src.comp( 0 ), src.comp( 1 ), src.comp( 2 ) };
        T*       d[3];
        dst.ptrs( d );
        if constexpr ( std::is_same_v< T, double > )
            check( tn_restriction_constant_f64( f_.get(), c_.get(), 3, s, d, stream() ), "restriction" );
        else
            check( tn_restriction_constant_f32( f_.get(), c_.get(), 3, s, d, stream() ), "restriction" );
    }

  private:
    Mesh f_, c_;
};

// KMass (kmass.hpp:17): mode 0 consistent, 1 diagonal, 2 lumped
template < typename T >
class KMass
{
  public:
    using SrcVectorType = VectorQ1Scalar< T >;
    using DstVectorType = VectorQ1Scalar< T >;
    using ScalarType    = T;
    KMass() = default;
    KMass( const Mesh& mesh, const VectorQ1Scalar< T >& k, int mode ) : mesh_( mesh ), k_( k ), mode_( mode ) {}
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        if constexpr ( std::is_same_v< T, double > )
            check( tn_kmass_apply_f64( mesh_.get(), k_.comp( 0 ), mode_, TN_APPLY_REPLACE, TN_COMM_ADDITIVE,
                                       src.comp( 0 ), dst.comp( 0 ), stream() ),
                   "kmass apply" );
        else
            check( tn_kmass_apply_f32( mesh_.get(), k_.comp( 0 ), mode_, TN_APPLY_REPLACE, TN_COMM_ADDITIVE,
                                       src.comp( 0 ), dst.comp( 0 ), stream() ),
                   "kmass apply" );
    }

  private:
    Mesh                mesh_;
    VectorQ1Scalar< T > k_;
    int                 mode_ = 0;
};

// VectorMass (vector_mass.hpp:17): the mass matrix (k = 1; full or diagonal)
// applied to each of the NC components (the reference's ViscousMass)
template < typename T, int NC = 3 >
class VectorMass
{
  public:
    using SrcVectorType = VectorQ1Base< T, NC >;
    using DstVectorType = VectorQ1Base< T, NC >;
    using ScalarType    = T;
    VectorMass() = default;
    VectorMass( const Mesh& mesh, bool diagonal ) : mesh_( mesh ), mode_( diagonal ? 1 : 0 ) {}
    void set_operator_apply_and_communication_modes( OperatorApplyMode am, OperatorCommunicationMode cm )
    {
        am_ = am, cm_ = cm;
    }
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        for ( int c = 0; c < NC; ++c )
        {
            if constexpr ( std::is_same_v< T, double > )
                check( tn_kmass_apply_f64( mesh_.get(), nullptr, mode_, int( am_ ), int( cm_ ), src.comp( c ),
                                           dst.comp( c ), stream() ),
                       "vector mass apply" );
            else
                check( tn_kmass_apply_f32( mesh_.get(), nullptr, mode_, int( am_ ), int( cm_ ), src.comp( c ),
                                           dst.comp( c ), stream() ),
                       "vector mass apply" );
        }
    }

  private:
    Mesh                      mesh_;
    int                       mode_ = 0;
    OperatorApplyMode         am_   = OperatorApplyMode::Replace;
    OperatorCommunicationMode cm_   = OperatorCommunicationMode::CommunicateAdditively;
};

// DiagonallyScaledOperator (linalg/diagonally_scaled_operator.hpp:15): D^{-1} A
// UnsteadyAdvectionDiffusionSUPG (unsteady_advection_diffusion_supg.hpp:134-420): the BDF left-hand side
// mass_scaling M + dt (K + C + G) with SUPG stabilisation for the velocity u
template < typename T >
class UnsteadyAdvectionDiffusionSUPG
{
  public:
    using SrcVectorType = VectorQ1Scalar< T >;
    using DstVectorType = VectorQ1Scalar< T >;
    using ScalarType    = T;
    UnsteadyAdvectionDiffusionSUPG( const Mesh& mesh, const VectorQ1Vec< T >& velocity, T diffusivity, T dt,
                                    bool treat_boundary, bool diagonal = false, T mass_scaling = T( 1 ),
                                    bool lumped_mass = false )
    : mesh_( mesh ), u_( velocity ), kappa_( diffusivity ), dt_( dt ), treat_( treat_boundary ), diag_( diagonal ),
      ms_( mass_scaling ), lumped_( lumped_mass )
    {}
    T&       dt() { return dt_; }
    const T& dt() const { return dt_; }
    void     set_operator_apply_and_communication_modes( OperatorApplyMode am, OperatorCommunicationMode cm )
    {
        am_ = am, cm_ = cm;
    }
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        const T* v[3] = { u_.comp( 0 ), u_.comp( 1 ), u_.comp( 2 ) };
        if constexpr ( std::is_same_v< T, double > )
            check( tn_supg_apply_f64( mesh_.get(), v, kappa_, dt_, ms_, lumped_, treat_, diag_, int( am_ ), int( cm_ ),
                                      src.comp( 0 ), dst.comp( 0 ), stream() ),
                   "supg apply" );
        else
            check( tn_supg_apply_f32( mesh_.get(), v, kappa_, dt_, ms_, lumped_, treat_, diag_, int( am_ ), int( cm_ ),
                                      src.comp( 0 ), dst.comp( 0 ), stream() ),
                   "supg apply" );
    }

  private:
    Mesh                      mesh_;
    VectorQ1Vec< T >          u_;
    T                         kappa_, dt_;
    bool                      treat_, diag_;
    T                         ms_;
    bool                      lumped_;
    OperatorApplyMode         am_ = OperatorApplyMode::Replace;
    OperatorCommunicationMode cm_ = OperatorCommunicationMode::CommunicateAdditively;
};

template < typename Op >
class DiagonallyScaledOperator
{
  public:
    using SrcVectorType = typename Op::SrcVectorType;
    using DstVectorType = typename Op::DstVectorType;
    using ScalarType    = typename Op::ScalarType;
    DiagonallyScaledOperator( Op& op, const SrcVectorType& inv_diag ) : op_( op ), inv_diag_( inv_diag ) {}
    void apply_impl( const SrcVectorType& src, DstVectorType& dst )
    {
        apply( op_, src, dst );
        scale_in_place( dst, inv_diag_ );
    }

  private:
    Op&           op_;
    SrcVectorType inv_diag_;
};

}  // namespace tn
