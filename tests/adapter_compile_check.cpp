// Compiled by tests/test_adapter_compiles.py against the reference's own headers: the adapter in
// include/vfb_virtualfluids_adapter.hpp must plug into KernelImp, BoundaryConditionFactory and
// GridScalingFactory unchanged. Every adapter entry is instantiated and assigned to the reference's
// own types.
#include "vfb_virtualfluids_adapter.hpp"

#include "Kernel/KernelFactory/KernelFactory.h"

using BCF = BoundaryConditionFactory;

void adapter_compile_check(std::shared_ptr<Parameter> para)
{
    std::shared_ptr<Kernel> k = vfb_adapter::make_kernel(para, "K17CompressibleNavierStokes", 0);
    std::shared_ptr<KernelImp> ki = vfb_adapter::K17CompressibleNavierStokesB200::getNewInstance(para, 0);
    k->run();
    k->runOnIndices(nullptr, 0u, CollisionTemplate::AllFeatures, CudaStreamIndex::Legacy);
    std::vector<PreProcessorType> pre = k->getPreProcessorTypes();
    (void)ki->getKernelUsesFluidNodeIndices();
    (void)pre;

    for (BCF::VelocityBC v : { BCF::VelocityBC::VelocityBounceBack, BCF::VelocityBC::VelocityInterpolatedIncompressible,
                               BCF::VelocityBC::VelocityInterpolatedCompressible,
                               BCF::VelocityBC::VelocityWithPressureInterpolatedCompressible }) {
        boundaryCondition bc = vfb_adapter::velocity_bc(v);
        (void)bc;
    }
    for (BCF::NoSlipBC v : { BCF::NoSlipBC::NoSlipDelayBounceBack, BCF::NoSlipBC::NoSlipBounceBack,
                             BCF::NoSlipBC::NoSlipInterpolatedIncompressible, BCF::NoSlipBC::NoSlipInterpolatedCompressible }) {
        boundaryCondition bc = vfb_adapter::noslip_bc(v, VFB_ARITH_FAST);
        (void)bc;
    }
    for (BCF::PressureBC v : { BCF::PressureBC::PressureNonEquilibriumIncompressible,
                               BCF::PressureBC::PressureNonEquilibriumCompressible, BCF::PressureBC::OutflowNonReflective,
                               BCF::PressureBC::OutflowNonReflectivePressureCorrection }) {
        boundaryConditionDirectional bc = vfb_adapter::pressure_bc(v, para.get());
        (void)bc;
    }
    vfb_adapter::BoundaryConditionFactoryB200 factory(BCF::VelocityBC::VelocityInterpolatedCompressible,
                                                      BCF::PressureBC::PressureNonEquilibriumCompressible, para.get());
    const BoundaryConditionFactory &base = factory;
    boundaryCondition velocity = base.getVelocityBoundaryConditionPost();
    std::variant<boundaryCondition, boundaryConditionDirectional> pressure = base.getPressureBoundaryConditionPre();
    (void)velocity;
    (void)pressure;

    gridScaling fc = vfb_adapter::scaling(true), cf = vfb_adapter::scaling(false);
    (void)fc;
    (void)cf;
    vfb_level L = vfb_adapter::level_of(*para, 0);
    (void)L;
    vfb_adapter::init_level(*para, 0);
    boundaryCondition slip = vfb_adapter::slip_bc(BCF::SlipBC::SlipCompressible);
    (void)slip;
}
