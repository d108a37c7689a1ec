// A host program written against the reference's call surface (as SU3_main.cpp uses it),
// compiled against include/lettuce_gpu.hpp instead of the reference headers.  Prints one
// line per measurement; tests/test_dropin.py compiles it (CPU) and runs it (GPU).
#include <cstdio>
#include <cstdlib>

#include "lettuce_gpu.hpp"

using namespace lettuce_gpu;

int main(int argc, char** argv)
{
    const int L = argc > 1 ? std::atoi(argv[1]) : 8;
    GaugeField Gluon({L, L, L, L});
    GaugeField Gluonsmeared1({L, L, L, L});
    Gluon.SetToHaarRandom(2024);

    auto& SimulatedAction = GaugeAction::WilsonAction;
    SimulatedAction.SetBeta(6.0);
    HeatbathKernel Heatbath(Gluon, SimulatedAction, 7);
    OverrelaxationSubgroupKernel OverrelaxationSubgroup(Gluon, SimulatedAction);
    for (int n = 0; n < 20; ++n)
    {
        Iterator::Checkerboard4(Heatbath, 1);
        Iterator::Checkerboard4(OverrelaxationSubgroup, 4);
    }
    std::printf("plaquette %.15f\n", PlaquetteSum(Gluon) / Gluon.Volume() / 18.0);
    std::printf("action %.12f\n", SimulatedAction.Action(Gluon));

    // the measurement bundle of the reference driver (SU3_main.cpp:117-139)
    GaugeAction::Rectangular<2> SymanzikAction(6.0, 1.0 + 8.0 / 12.0, -1.0 / 12.0);
    GaugeField Gluonchain({L, L, L, L});
    const std::complex<double> poly = PolyakovLoop(Gluon);
    double q_sum = 0.0;
    for (const double q : TopChargeCloverTimeslices(Gluon)) q_sum += q;
    // the chain grows from call to call, so the loops are evaluated in order (SU3_main.cpp:141-143)
    const double w2 = WilsonLoop<0, 2, true>(Gluon, Gluonchain);
    const double w4 = WilsonLoop<2, 4, false>(Gluon, Gluonchain);
    std::printf("bundle S %.15f W2 %.15f W4 %.15f P %.15f %.15f Qplaq %.15f Qt %.15f E0 %.15f\n",
                SymanzikAction.ActionNormalized(Gluon), w2, w4, poly.real(), poly.imag(), TopChargePlaquette(Gluon),
                q_sum, EnergyDensity::CloverTimeslice(Gluon, 0));
    Integrators::GradientFlow::Euler euler;
    GradientFlowKernel EulerFlow(Gluon, Gluonchain, euler, SimulatedAction, 0.02);
    EulerFlow(5);
    std::printf("euler E %.15f\n", EnergyDensityClover(Gluonchain));

    Integrators::GradientFlow::RK3 rk3;
    GradientFlowKernel Flow(Gluon, Gluonsmeared1, rk3, SimulatedAction, 0.01);
    Flow(10);
    for (int m = 0; m < 3; ++m)
    {
        Flow.Resume(10);
        std::printf("flow t=%.2f Q %.12f E %.12f\n", 0.1 * (m + 2), TopChargeClover(Gluonsmeared1),
                    EnergyDensityClover(Gluonsmeared1));
    }

    // the clover field as a FullTensor (CalculateClover<1, 1>) and Q from it
    FullTensor Clover(Gluon.Shape());
    CalculateClover(Gluon, Clover);
    std::printf("tensor Q %.15f %.15f\n", TopChargeClover(Clover), TopChargeClover(Gluon));

    // the Zeuthen flow as the flow's action (no counterpart in the reference)
    GradientFlowKernel ZeuthenFlow(Gluon, Gluonchain, rk3, GaugeAction::ZeuthenFlowAction, 0.01);
    ZeuthenFlow(10);
    std::printf("zeuthen E %.15f\n", EnergyDensityClover(Gluonchain));

    // the reference driver's HMC integrator, OMF_4 (SU3_main.cpp:331), then a parity update (:527-531)
    Integrators::HMC::OMF_4 omf4;
    RunStatistics hmc_statistics;
    GaugeUpdates::HMCKernel HMC(Gluon, omf4, SimulatedAction, hmc_statistics, 1.0, 5);
    HMC(10, false);
    const double q_before = TopChargeClover(Gluon);
    ParityUpdate(Gluon, Gluonsmeared1);
    std::printf("parity dH %.10f Q %.12f %.12f\n", hmc_statistics.delta_H_hmc, q_before, TopChargeClover(Gluon));

    MetaBiasPotential TopBiasPotential(-8.0, 8.0, 800, 0.05, 4 * 16.0 / 800, 10.0, 1000.0);
    TopBiasPotential.SetUpdateMode(LT_BIAS_BINNED);
    RunStatistics statistics;
    Integrators::HMC::OMF_2_OMF_4 omf2_omf4;
    GaugeUpdates::HMCMetaDKernel HMC_MetaD(Gluon, TopBiasPotential, omf2_omf4, SimulatedAction, statistics, 1.0, 0.12, 4, 99);
    for (int n = 0; n < 3; ++n)
    {
        bool acc = HMC_MetaD(10, true);
        std::printf("metad dH %.10f accepted %d cv %.10f\n", statistics.delta_H_hmc, acc ? 1 : 0, HMC_MetaD.cv_current);
    }
    GaugeField copy(Gluon);
    Swap(copy, Gluonsmeared1);
    std::printf("copy plaquette %.15f\n", PlaquetteSum(Gluonsmeared1) / Gluon.Volume() / 18.0);

    // checkpoints as the reference's driver writes them (CheckpointManager + BMW files)
    if (argc > 2)
    {
        CheckpointManager checkpoints(argv[2], 3, true);
        for (int k = 0; k < 3; ++k)
        {
            Iterator::Checkerboard4(Heatbath, 1);
            checkpoints.AlternatingCheckpoints(SaveConfigBMWFull, Heatbath, Gluon, "config", "prng_state", "distribution_state");
        }
        GaugeField restored({L, L, L, L});
        HeatbathKernel resumed(restored, SimulatedAction);
        checkpoints.LoadCheckpoint(LoadConfigBMWFull, resumed, restored, "config", "prng_state", "distribution_state");
        bool checksum_ok = false;
        const bool in_group = LoadConfigBMWChecked(restored, (checkpoints.CheckpointDirectory() / "missing").string(),
                                                   false, checksum_ok);
        std::printf("checkpoint counter %llu restored plaquette %.15f original %.15f missing %d\n",
                    (unsigned long long)resumed.counter, PlaquetteSum(restored) / Gluon.Volume() / 18.0,
                    PlaquetteSum(Gluon) / Gluon.Volume() / 18.0, in_group ? 1 : 0);
    }
    return 0;
}
