/*
 * ref_main_cuda.cc -- the reference's driver flow (src/Main.cc:186-360) with
 * the GPU sweeper plugged in through tycho2_b200/csrc/SweeperCuda.hh: the
 * reference's own deck reader, quadrature, TychoMesh, cross sections,
 * Problem and .psi writer, with SweeperCuda in place of SweeperTraverse.
 * It is what a maintainer gets after adding `SweepType Cuda` to the
 * reference; built against the reference sources by oracle/Makefile and
 * used by the GPU tests to show the drop-in reproduces gold.psi.
 *
 *   sweep_cuda.x <pmesh> <deck> [reference-loop]
 *
 * Default: SweeperCuda::solve (the outer iteration resident on the device).
 * With `reference-loop` (decks with SourceIteration true): the reference's
 * own SourceIteration::fixedPoint drives SweeperCuda::sweep, exactly as
 * SweeperTraverse::solve drives SweeperTraverse::sweep
 * (src/SweeperTraverse.cc:65-74, src/SourceIteration.cc:127-207), with the
 * reference's PsiData containers (host `new double[]` buffers) handed to
 * the GPU sweep at every iteration.
 */
#include <cstdio>
#include <string>

#include <mpi.h>

#include "Global.hh"
#include "KeyValueReader.hh"
#include "Problem.hh"
#include "PsiData.hh"
#include "Quadrature.hh"
#include "SourceIteration.hh"
#include "TychoMesh.hh"
#include "SweeperCuda.hh"

int main(int argc, char **argv)
{
    if (argc < 3) {
        printf("Usage: ./sweep_cuda.x <parallel mesh> <input deck> [reference-loop]\n");
        return 0;
    }
    const bool reference_loop = argc > 3 && std::string(argv[3]) == "reference-loop";
    int provided = 0;
    MPI_Init_thread(&argc, &argv, MPI_THREAD_SINGLE, &provided);
    CKG_Utils::KeyValueReader kvr;
    kvr.readFile(argv[2]);
    int snOrder, iterMax, nGroups;
    double sigmaT1, sigmaS1, sigmaT2, sigmaS2;
    std::string gauss;
    kvr.getInt("snOrder", snOrder);
    kvr.getInt("iterMax", iterMax);
    kvr.getDouble("errMax", g_errMax);
    kvr.getInt("nGroups", nGroups);
    kvr.getDouble("sigmaT1", sigmaT1);
    kvr.getDouble("sigmaS1", sigmaS1);
    kvr.getDouble("sigmaT2", sigmaT2);
    kvr.getDouble("sigmaS2", sigmaS2);
    kvr.getBool("OutputFile", g_outputFile);
    kvr.getString("OutputFilename", g_outputFilename);
    kvr.getBool("SourceIteration", g_useSourceIteration);
    kvr.getString("GaussElim", gauss);
    g_snOrder = snOrder;
    g_iterMax = iterMax;
    g_nGroups = nGroups;
    // the deck key as src/Main.cc:167-176 reads it (NoPivot if absent)
    g_gaussElim = gauss == "Original"      ? GaussElim_Original
                  : gauss == "CramerGlu"   ? GaussElim_CramerGlu
                  : gauss == "CramerIntel" ? GaussElim_CramerIntel
                                           : GaussElim_NoPivot;
    g_nAngleGroups = g_nThreads = 1;
    g_quadrature = new Quadrature(g_snOrder);
    g_tychoMesh = new TychoMesh(argv[1]);
    Problem::createCrossSections(g_sigmaT, g_sigmaS, sigmaT1, sigmaS1, sigmaT2, sigmaS2);

    SweeperCuda sweeper;
    if (reference_loop) {
        Insist(g_useSourceIteration, "reference-loop runs SourceIteration::fixedPoint (SourceIteration true)");
        // as SweeperTraverse::solve: the sweeper's own psi, a fixed source
        PsiData &psi = sweeper.getPsi();
        PsiData source;
        Problem::getSource(source);
        psi.setToValue(0.0);
        const UINT iters = SourceIteration::fixedPoint(sweeper, psi, source);
        printf("reference fixedPoint over SweeperCuda::sweep: %llu iterations\n", (unsigned long long)iters);
        printf("L2 Relative Error: %e\n", Problem::hatL2Error(psi));
        if (g_outputFile) psi.writeToFile(g_outputFilename);
    } else {
        sweeper.solve();
        printf("L2 Relative Error: %e\n", Problem::hatL2Error(sweeper.getPsi()));
        if (g_outputFile) sweeper.writePsiToFile(g_outputFilename);
    }
    MPI_Finalize();
    return 0;
}
