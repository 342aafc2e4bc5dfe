/*
 * ref_main_cuda.cc -- the reference's driver flow (src/Main.cc:186-360) with
 * the GPU sweeper plugged in through tycho2_b200/csrc/SweeperCuda.hh: the
 * reference's own deck reader, quadrature, TychoMesh, cross sections,
 * Problem and .psi writer, with SweeperCuda in place of SweeperTraverse.
 * It is what a maintainer gets after adding `SweepType Cuda` to the
 * reference; built against the reference sources by oracle/Makefile and
 * used by the GPU tests to show the drop-in reproduces gold.psi.
 *
 *   sweep_cuda.x <pmesh> <deck>
 */
#include <cstdio>
#include <string>

#include <mpi.h>

#include "Global.hh"
#include "KeyValueReader.hh"
#include "Problem.hh"
#include "Quadrature.hh"
#include "TychoMesh.hh"
#include "SweeperCuda.hh"

int main(int argc, char **argv)
{
    if (argc < 3) {
        printf("Usage: ./sweep_cuda.x <parallel mesh> <input deck>\n");
        return 0;
    }
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
    g_gaussElim = gauss == "Original" ? GaussElim_Original : GaussElim_NoPivot;
    g_nAngleGroups = g_nThreads = 1;
    g_quadrature = new Quadrature(g_snOrder);
    g_tychoMesh = new TychoMesh(argv[1]);
    Problem::createCrossSections(g_sigmaT, g_sigmaS, sigmaT1, sigmaS1, sigmaT2, sigmaS2);

    SweeperCuda sweeper;
    sweeper.solve();
    printf("L2 Relative Error: %e\n", Problem::hatL2Error(sweeper.getPsi()));
    if (g_outputFile) sweeper.writePsiToFile(g_outputFilename);
    MPI_Finalize();
    return 0;
}
