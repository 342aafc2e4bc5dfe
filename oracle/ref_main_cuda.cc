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
 *   sweep_cuda.x <pmesh> <deck> sweep-local <sigmaT.f64> <source.f64> <psiBound.f64> <out.f64>
 *
 * Default: SweeperCuda::solve (the outer iteration resident on the device).
 * With `reference-loop` (decks with SourceIteration true): the reference's
 * own SourceIteration::fixedPoint drives SweeperCuda::sweep, exactly as
 * SweeperTraverse::solve drives SweeperTraverse::sweep
 * (src/SweeperTraverse.cc:65-74, src/SourceIteration.cc:127-207), with the
 * reference's PsiData containers (host `new double[]` buffers) handed to
 * the GPU sweep at every iteration.
 * With `sweep-local`: one rank's partition (TYCHO_SHIM_RANK of
 * TYCHO_SHIM_SIZE, oracle/ref_shim/mpi.h), per-cell sigma_t, an angular
 * source and psiBound read from files, one SweeperCuda::sweepLocal -- what
 * src/Util.cc:138-145 becomes with the GPU -- and psi written to <out.f64>.
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
    const bool sweep_local = argc == 8 && std::string(argv[3]) == "sweep-local";
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
    if (sweep_local) {
        auto load = [](const char *path, double *dst, size_t n) {
            FILE *fp = fopen(path, "rb");
            Insist(fp && fread(dst, sizeof(double), n, fp) == n, "cannot read an input file");
            fclose(fp);
        };
        load(argv[4], g_sigmaT.data(), g_nCells);
        for (UINT c = 0; c < g_nCells; c++) g_sigmaS[c] = 0.0;
        SweeperCuda sweeper;
        PsiData source, psi;
        PsiBoundData psiBound;
        load(argv[5], &source[0], source.size());
        load(argv[6], &psiBound[0], psiBound.size());
        sweeper.sweepLocal(psi, source, psiBound);
        FILE *fp = fopen(argv[7], "wb");
        Insist(fp && fwrite(&psi[0], sizeof(double), psi.size(), fp) == psi.size(), "cannot write psi");
        fclose(fp);
        MPI_Finalize();
        return 0;
    }

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
