/*
 * The VirtualFluids side of the binding: what a maintainer adds to the reference tree so that its
 * GPU time step calls this library. Header-only C++; it includes the reference's own headers
 * (src/gpu/core/Kernel/KernelImp.h, Parameter/Parameter.h, BoundaryConditions/
 * BoundaryConditionFactory.h, GridScaling/GridScalingFactory.h) and the C ABI (vfb.h), and it
 * changes nothing in the reference: it plugs into its extension points.
 *
 *  - vfb_level_of(para, level) / vfb_level_of(LBMSimulationParameter*): the level view the ABI takes,
 *    read from the fields the reference already keeps (Parameter.h:66-330).
 *  - K17CompressibleNavierStokesB200: a KernelImp (Kernel/Kernel.h:44-51) for the name
 *    "K17CompressibleNavierStokes", to return from KernelFactoryImp::makeKernel
 *    (Kernel/KernelFactory/KernelFactoryImp.cpp:92-139) in place of K17CompressibleNavierStokes<None>.
 *  - vfb_velocity_bc / vfb_noslip_bc / vfb_pressure_bc: the std::function values that the
 *    getters of BoundaryConditionFactory (BoundaryConditionFactory.cpp:85-219) return for each enum
 *    value; BoundaryConditionFactoryB200 overrides the two virtual getters with them.
 *  - vfb_scaling_fine_to_coarse / vfb_scaling_coarse_to_fine: the gridScaling functions
 *    (GridScaling/GridScalingFactory.h:46) for GridScaling::ScaleCompressible.
 *
 * Errors: the ABI returns status codes; the adapter turns them into std::runtime_error, the way the
 * reference reports configuration errors. The ABI allocates nothing and never takes ownership of
 * the reference's buffers; the BC and scaling functions run on the legacy stream, as the
 * reference's own kernels do.
 */
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <variant>

#include "BoundaryConditions/BoundaryConditionFactory.h"
#include "Calculation/Calculation.h"
#include "GridScaling/GridScalingFactory.h"
#include "Kernel/KernelImp.h"
#include "Parameter/Parameter.h"
#include "vfb.h"

namespace vfb_adapter
{

//! status of an ABI call as the reference reports errors
inline void check(int status)
{
    if (status != VFB_OK)
        throw std::runtime_error(std::string("virtualfluids_b200: ") + vfb_last_error());
}

//! the storage the reference's `real` maps to (basics/DataTypes.h:39-43)
constexpr int32_t real_storage() { return sizeof(real) == 8 ? VFB_STORAGE_F64 : VFB_STORAGE_F32; }

//! the level fields every entry point reads, from one LBMSimulationParameter (device side)
inline vfb_level level_of(const LBMSimulationParameter *p, int level_index, int32_t arith = VFB_ARITH_EXACT)
{
    vfb_level L{};
    L.storage = real_storage();
    L.arith = arith;
    L.is_even_timestep = p->isEvenTimestep ? 1 : 0;
    L.level = level_index;
    L.number_of_nodes = p->numberOfNodes;
    L.distributions = p->distributions.f[0];
    L.neighbor_x = p->neighborX;
    L.neighbor_y = p->neighborY;
    L.neighbor_z = p->neighborZ;
    L.type_of_grid_node = p->typeOfGridNode;
    L.omega = p->omega;
    L.rho = p->rho;
    L.velocity_x = p->velocityX;
    L.velocity_y = p->velocityY;
    L.velocity_z = p->velocityZ;
    L.pressure = p->pressure;
    L.body_force_x = p->forceX_SP;
    L.body_force_y = p->forceY_SP;
    L.body_force_z = p->forceZ_SP;
    for (int i = 0; i < 3; ++i)
        L.quadric_limiters[i] = 0.01;       // Parameter.cpp:69 default; vfb_level_of(para, ...) reads the set value
    return L;
}

//! the same with the Parameter-wide values: forcing, quadric limiters, outflow correction factor
inline vfb_level level_of(Parameter &para, int level_index, int32_t arith = VFB_ARITH_EXACT)
{
    vfb_level L = level_of(para.getParD(level_index).get(), level_index, arith);
    for (int i = 0; i < 3; ++i) {
        L.forces[i] = para.getForcesDouble()[i];
        L.quadric_limiters[i] = para.getQuadricLimitersDouble()[i];
    }
    L.outflow_pressure_correction_factor = para.getOutflowPressureCorrectionFactor();
    return L;
}

//! InitNavierStokesCompressible::init (InitNavierStokesCompressible.cu:45-84) of one level at its
//! current parity: the non-equilibrium init from the velocity gradients when
//! Parameter::getUseInitNeq() is set (it reads neighborInverse), else the equilibrium
inline void init_level(Parameter &para, int level_index, int32_t arith = VFB_ARITH_EXACT)
{
    const vfb_level L = level_of(para, level_index, arith);
    if (para.getUseInitNeq())
        check(vfb_init_navier_stokes_compressible_non_equilibrium(&L, para.getParD(level_index)->neighborInverse,
                                                                  nullptr));
    else
        check(vfb_init_navier_stokes_compressible(&L, nullptr));
}

//! QforBoundaryConditions (Calculation.h:105-117) as the ABI's vfb_bc
inline vfb_bc bc_of(const QforBoundaryConditions *q)
{
    vfb_bc b{};
    b.k = q->k;
    b.q27 = q->q27[0];
    b.number_of_bc_nodes = q->numberOfBCnodes;
    b.vx = q->Vx;
    b.vy = q->Vy;
    b.vz = q->Vz;
    return b;
}

//! QforDirectionalBoundaryCondition (Calculation.h:119-127) as the ABI's vfb_directional_bc
inline vfb_directional_bc directional_bc_of(const QforDirectionalBoundaryCondition *q)
{
    vfb_directional_bc b{};
    b.k = q->k;
    b.k_neighbor = q->kN;
    b.rho_bc = q->RhoBC;
    b.number_of_bc_nodes = q->numberOfBCnodes;
    b.direction = static_cast<int32_t>(q->direction);
    return b;
}

// ---------------------------------------------------------------------------------------------
// collision kernel: K17CompressibleNavierStokes<TurbulenceModel::None>
// ---------------------------------------------------------------------------------------------
class K17CompressibleNavierStokesB200 : public KernelImp
{
public:
    static std::shared_ptr<K17CompressibleNavierStokesB200> getNewInstance(std::shared_ptr<Parameter> para, int level)
    {
        return std::shared_ptr<K17CompressibleNavierStokesB200>(new K17CompressibleNavierStokesB200(para, level));
    }

    //! K17CompressibleNavierStokes.cu:85-100: the default template over the tagged fluid nodes
    void run() override
    {
        LBMSimulationParameter *p = para->getParD(level).get();
        runOnIndices(p->taggedFluidNodeIndices[CollisionTemplate::Default],
                     p->numberOfTaggedFluidNodes[CollisionTemplate::Default], CollisionTemplate::Default,
                     CudaStreamIndex::Legacy);
    }

    //! K17CompressibleNavierStokes.cu:102-145: every CollisionTemplate, on the stream of the index.
    //! Each index list gets a prepared plan on its first call (its slot table, and box addressing for
    //! a regular periodic box); the reference sets its lists and neighbour arrays up once. After
    //! changing them, call invalidatePlans().
    void runOnIndices(const unsigned int *indices, unsigned int size_indices, CollisionTemplate collisionTemplate,
                      CudaStreamIndex streamIndex = CudaStreamIndex::Legacy) override
    {
        vfb_level L = level_of(*para, level, arith);
        vfb_k17_plan *&plan = plans[{ indices, size_indices }];
        if (!plan)
            check(vfb_k17_plan_create(&L, indices, size_indices, &plan));
        check(vfb_k17_plan_run(plan, &L, static_cast<int32_t>(collisionTemplate),
                               para->getStreamManager()->getStream(streamIndex)));
    }

    void invalidatePlans()
    {
        for (auto &kv : plans)
            vfb_k17_plan_destroy(kv.second);
        plans.clear();
    }
    ~K17CompressibleNavierStokesB200() override { invalidatePlans(); }

    //! VFB_ARITH_EXACT (default): the reference's rounding bit for bit; VFB_ARITH_FAST: FMA arithmetic
    void setArithmetic(int32_t a) { arith = a; }

private:
    K17CompressibleNavierStokesB200(std::shared_ptr<Parameter> p, int l) : KernelImp(p, l)
    {
        // as K17CompressibleNavierStokes.cu:147-156
        myPreProcessorTypes.push_back(InitNavierStokesCompressible);
        kernelUsesFluidNodeIndices = true;
    }
    int32_t arith = VFB_ARITH_EXACT;
    std::map<std::pair<const unsigned int *, unsigned int>, vfb_k17_plan *> plans;
};

//! KernelFactoryImp::makeKernel's branch for the name (the reference throws for unknown names;
//! vfb_kernel_lookup answers VFB_ERR_UNKNOWN_KERNEL for them)
inline std::shared_ptr<Kernel> make_kernel(std::shared_ptr<Parameter> para, const std::string &kernel, int level)
{
    int32_t id = 0;
    if (vfb_kernel_lookup(kernel.c_str(), &id) != VFB_OK)
        throw std::runtime_error("KernelFactory does not know the KernelType.");
    return K17CompressibleNavierStokesB200::getNewInstance(para, level);
}

// ---------------------------------------------------------------------------------------------
// boundary conditions (BoundaryConditionFactory.cpp:85-219)
// ---------------------------------------------------------------------------------------------
using bc_entry = int (*)(const vfb_level *, const vfb_bc *, void *);
using directional_bc_entry = int (*)(const vfb_level *, const vfb_directional_bc *, void *);

inline boundaryCondition bind_bc(bc_entry fn, int32_t arith)
{
    return [fn, arith](LBMSimulationParameter *p, QforBoundaryConditions *q) {
        const vfb_level L = level_of(p, 0, arith);
        const vfb_bc b = bc_of(q);
        check(fn(&L, &b, nullptr));
    };
}

//! getVelocityBoundaryConditionPost for each VelocityBC value (an empty function for NotSpecified,
//! which the reference's BoundaryConditionKernelManager rejects when the BC has nodes)
inline boundaryCondition velocity_bc(BoundaryConditionFactory::VelocityBC v, int32_t arith = VFB_ARITH_EXACT)
{
    switch (v) {
    case BoundaryConditionFactory::VelocityBC::VelocityBounceBack:
        return bind_bc(vfb_velocity_bounce_back, arith);
    case BoundaryConditionFactory::VelocityBC::VelocityInterpolatedIncompressible:
        return bind_bc(vfb_velocity_interpolated_incompressible, arith);
    case BoundaryConditionFactory::VelocityBC::VelocityInterpolatedCompressible:
        return bind_bc(vfb_velocity_interpolated_compressible, arith);
    case BoundaryConditionFactory::VelocityBC::VelocityWithPressureInterpolatedCompressible:
        return bind_bc(vfb_velocity_with_pressure_interpolated_compressible, arith);
    default:
        return nullptr;
    }
}

//! getNoSlipBoundaryConditionPost for each NoSlipBC value; the delayed bounce-back is the
//! deliberately empty function (the esoteric twist with links to the dummy node)
inline boundaryCondition noslip_bc(BoundaryConditionFactory::NoSlipBC v, int32_t arith = VFB_ARITH_EXACT)
{
    switch (v) {
    case BoundaryConditionFactory::NoSlipBC::NoSlipDelayBounceBack:
        return [](LBMSimulationParameter *, QforBoundaryConditions *) {};
    case BoundaryConditionFactory::NoSlipBC::NoSlipBounceBack:
        return bind_bc(vfb_noslip_bounce_back, arith);
    case BoundaryConditionFactory::NoSlipBC::NoSlipInterpolatedIncompressible:
        return bind_bc(vfb_noslip_interpolated_incompressible, arith);
    case BoundaryConditionFactory::NoSlipBC::NoSlipInterpolatedCompressible:
        return bind_bc(vfb_noslip_interpolated_compressible, arith);
    }
    return nullptr;
}

//! getSlipBoundaryConditionPost for each SlipBC value (not virtual in the reference: its switch in
//! BoundaryConditionFactory.cpp returns slip_bc(...)); the turbulent-viscosity form stays the
//! reference's, as it reads the turbulence model's viscosity
inline boundaryCondition slip_bc(BoundaryConditionFactory::SlipBC v, int32_t arith = VFB_ARITH_EXACT)
{
    if (v == BoundaryConditionFactory::SlipBC::SlipCompressible)
        return bind_bc(vfb_slip_compressible, arith);
    return nullptr;
}

//! getPressureBoundaryConditionPre for each PressureBC value (the directional form every
//! implemented pressure kernel takes). The outflow with pressure correction reads its factor from
//! the level view, so it binds the Parameter.
inline boundaryConditionDirectional pressure_bc(BoundaryConditionFactory::PressureBC v, Parameter *para,
                                                int32_t arith = VFB_ARITH_EXACT)
{
    directional_bc_entry fn = nullptr;
    switch (v) {
    case BoundaryConditionFactory::PressureBC::PressureNonEquilibriumIncompressible:
        fn = vfb_pressure_non_equilibrium_incompressible;
        break;
    case BoundaryConditionFactory::PressureBC::PressureNonEquilibriumCompressible:
        fn = vfb_pressure_non_equilibrium_compressible;
        break;
    case BoundaryConditionFactory::PressureBC::OutflowNonReflective:
        fn = vfb_outflow_non_reflecting;
        break;
    case BoundaryConditionFactory::PressureBC::OutflowNonReflectivePressureCorrection:
        fn = vfb_outflow_non_reflecting_pressure_correction;
        break;
    default:
        return nullptr;
    }
    return [fn, para, arith](LBMSimulationParameter *p, QforDirectionalBoundaryCondition *q) {
        vfb_level L = level_of(p, 0, arith);
        if (para)
            L.outflow_pressure_correction_factor = para->getOutflowPressureCorrectionFactor();
        const vfb_directional_bc b = directional_bc_of(q);
        check(fn(&L, &b, nullptr));
    };
}

//! the factory with the two virtual getters answered by the library; the no-slip getter is not
//! virtual in the reference, so its switch returns noslip_bc(...) in BoundaryConditionFactory.cpp
class BoundaryConditionFactoryB200 : public BoundaryConditionFactory
{
public:
    BoundaryConditionFactoryB200(VelocityBC velocity, PressureBC pressure, Parameter *para)
        : velocity(velocity), pressure(pressure), para(para)
    {
        setVelocityBoundaryCondition(velocity);
        setPressureBoundaryCondition(pressure);
    }
    [[nodiscard]] boundaryCondition getVelocityBoundaryConditionPost(bool isGeometryBC = false) const override
    {
        (void)isGeometryBC;
        return velocity_bc(velocity);
    }
    [[nodiscard]] std::variant<boundaryCondition, boundaryConditionDirectional> getPressureBoundaryConditionPre() const override
    {
        return pressure_bc(pressure, para);
    }

private:
    VelocityBC velocity;
    PressureBC pressure;
    Parameter *para;
};

// ---------------------------------------------------------------------------------------------
// grid scaling (GridScaling/GridScalingFactory.h:46, GridScaling::ScaleCompressible)
// ---------------------------------------------------------------------------------------------
inline vfb_interpolation_cells cells_of(const ICells *c)
{
    vfb_interpolation_cells out{};
    out.fine_cell_indices = c->fineCellIndices;
    out.coarse_cell_indices = c->coarseCellIndices;
    out.number_of_cells = c->numberOfCells;
    return out;
}

inline vfb_interpolation_cell_neighbor offsets_of(const ICellNeigh &n)
{
    vfb_interpolation_cell_neighbor out{};
    out.x = n.x;
    out.y = n.y;
    out.z = n.z;
    return out;
}

inline gridScaling scaling(bool fine_to_coarse, int32_t arith = VFB_ARITH_EXACT)
{
    return [fine_to_coarse, arith](LBMSimulationParameter *coarse, LBMSimulationParameter *fine, ICells *cells,
                                   ICellNeigh &neighbor, CUstream_st *stream) {
        const vfb_level C = level_of(coarse, 0, arith), F = level_of(fine, 1, arith);
        const vfb_interpolation_cells ic = cells_of(cells);
        const vfb_interpolation_cell_neighbor off = offsets_of(neighbor);
        check(fine_to_coarse ? vfb_scale_fine_to_coarse_compressible(&C, &F, &ic, &off, stream)
                             : vfb_scale_coarse_to_fine_compressible(&C, &F, &ic, &off, stream));
    };
}

} // namespace vfb_adapter
