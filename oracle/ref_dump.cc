/*
 * ref_dump.cc -- a driver that links the reference tycho2 sources, compiled
 * unmodified from their own tree by oracle/Makefile, and dumps what the
 * reference computes so that the C restatement (tycho_oracle.c) and through
 * it the B200 sweep can be pinned to it.  TEST INFRASTRUCTURE ONLY.
 *
 * Modes (all binary outputs are raw little-endian arrays):
 *   tables <pmesh> <snOrder> <outprefix>
 *       adjCell, neighborVrtx, faceToCellVrtx, cellToFaceVrtx (u64),
 *       volume, faceArea, omegaDotN (f64), initial dependency counts from the
 *       GraphTraverser constructor and b-levels from Priorities (u64).
 *   sweep <pmesh> <snOrder> <nGroups> <sigmaT.f64> <source.f64> <out.f64>
 *       one SweeperTraverse::sweep of an angular source (psi layout).
 *   si <pmesh> <snOrder> <nGroups> <sigmaT.f64> <sigmaS.f64> <source.f64>
 *      <iterMax> <errMax> <out.f64>
 *       SourceIteration::fixedPoint with per-cell sigma_t/sigma_s.
 *   levels <pmesh> <snOrder> <out.u64>
 *       SweepSchedule's b-levels: calcDependencies and calcLevels
 *       (src/SweepSchedule.cc:107-125, :472-508; the +-1e-10 omega.n rule)
 *       over every angle, (angle, cell) order, followed by their count.
 *   sweep_local <pmesh> <snOrder> <nGroups> <sigmaT.f64> <source.f64> <psiBound.f64>
 *               <out.f64> <outprefix>
 *       one rank's partition (TYCHO_SHIM_RANK of TYCHO_SHIM_SIZE, see
 *       ref_shim/mpi.h): Util::sweepLocal(psi, source, psiBound) under a
 *       GraphTraverser without communication, as the PBJ and Schur sweepers
 *       build it (src/Main.cc:283-315, src/Util.cc:138-145); psiBound in
 *       PsiBoundData layout (nSides, A, 3, G).  Also dumps the partition's
 *       adjCell, adjRank, side (u64, (c,4)) and lGSides (u64, nSides).
 *   bench <pmesh> <snOrder> <nGroups> <sigmaT.f64> <qiso.f64> <steps> <warmup> [<phi.f64>]
 *       times SweeperTraverse::sweep of an isotropic source on all OpenMP
 *       threads; prints REFBENCH with a hash of the last psi's bytes and,
 *       given <phi.f64>, writes Util::psiToPhi of that psi.
 *
 * The psi hash: the psi array read as 64-bit words x_i, sum of x_i * (2i+1)
 * modulo 2^64.  Equal hashes of two arrays of the same length mean equal
 * bits (up to a 2^-64 chance); the sum is order-free, so a caller can form
 * it in chunks or in parallel.
 */
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include <omp.h>

#include <map>
#include <mpi.h>
/* The initial dependency counts live in a private member; expose it for the
   dump only (the reference file itself is compiled unmodified elsewhere). */
#define private public
#include "GraphTraverser.hh"
#undef private
#include "Global.hh"
#include "Quadrature.hh"
#include "TychoMesh.hh"
#include "PsiData.hh"
#include "SweepData.hh"
#include "SourceIteration.hh"
#include "Priorities.hh"
#include "SweeperTraverse.hh"
#include "Util.hh"
/* calcDependencies and calcLevels are file-static in the reference: its
   SweepSchedule translation unit is compiled into this driver (and left out
   of the driver's link line) so that the dump calls the reference's own
   functions. */
#include "SweepSchedule.cc"

static void dump_u64(const std::string &path, const std::vector<UINT> &v)
{
    FILE *fp = fopen(path.c_str(), "wb");
    fwrite(v.data(), sizeof(UINT), v.size(), fp);
    fclose(fp);
}

static void dump_f64(const std::string &path, const double *v, size_t n)
{
    FILE *fp = fopen(path.c_str(), "wb");
    fwrite(v, sizeof(double), n, fp);
    fclose(fp);
}

static std::vector<double> load_f64(const std::string &path, size_t n)
{
    std::vector<double> v(n);
    FILE *fp = fopen(path.c_str(), "rb");
    if (!fp || fread(v.data(), sizeof(double), n, fp) != n) {
        fprintf(stderr, "ref_dump: cannot read %zu doubles from %s\n", n, path.c_str());
        exit(2);
    }
    fclose(fp);
    return v;
}

static void setup(const char *pmesh, int sn, int groups, bool comm = true)
{
    g_nAngleGroups = 1;
    #pragma omp parallel
    {
        if (omp_get_thread_num() == 0) g_nAngleGroups = omp_get_num_threads();
    }
    g_nThreads = g_nAngleGroups;
    g_snOrder = sn;
    g_nGroups = groups;
    g_maxCellsPerStep = 100;
    g_intraAngleP = 1;   /* b-level priorities: priorities == b-levels */
    g_interAngleP = 0;   /* interleaved: no per-angle offset */
    g_gaussElim = GaussElim_NoPivot;
    if (const char *ge = getenv("TYCHO_GAUSS_ELIM")) {  // deck key GaussElim
        std::string k = ge;
        g_gaussElim = k == "Original" ? GaussElim_Original
                      : k == "CramerGlu" ? GaussElim_CramerGlu
                      : k == "CramerIntel" ? GaussElim_CramerIntel
                                           : GaussElim_NoPivot;
    }
    g_mpiType = MPIType_TychoTwoSided;
    g_sweepType = SweepType_TraverseGraph;
    g_quadrature = new Quadrature(g_snOrder);
    g_tychoMesh = new TychoMesh(pmesh);
    g_graphTraverserForward =
        new GraphTraverser(Direction_Forward, comm, SweepData::getDataSizeInBytes());
}

int main(int argc, char **argv)
{
    if (argc < 2) return 2;
    std::string mode = argv[1];
    if (mode == "tables" && argc == 5) {
        setup(argv[2], atoi(argv[3]), 1);
        std::string pre = argv[4];
        UINT nc = g_nCells, na = g_nAngles;
        std::vector<UINT> adj(nc * 4), nbr(nc * 12), f2c(nc * 12), c2f(nc * 16, UINT64_MAX);
        std::vector<double> vol(nc), area(nc * 4), odn(na * nc * 4);
        for (UINT c = 0; c < nc; c++) {
            vol[c] = g_tychoMesh->getCellVolume(c);
            for (UINT f = 0; f < 4; f++) {
                adj[c * 4 + f] = g_tychoMesh->getAdjCell(c, f);
                area[c * 4 + f] = g_tychoMesh->getFaceArea(c, f);
                for (UINT k = 0; k < 3; k++) {
                    nbr[(c * 4 + f) * 3 + k] = g_tychoMesh->getNeighborVrtx(c, f, k);
                    f2c[(c * 4 + f) * 3 + k] = g_tychoMesh->getFaceToCellVrtx(c, f, k);
                }
                for (UINT v = 0; v < 4; v++)
                    if (v != f) c2f[(c * 4 + f) * 4 + v] = g_tychoMesh->getCellToFaceVrtx(c, f, v);
                for (UINT a = 0; a < na; a++)
                    odn[(f * nc + c) * na + a] = g_tychoMesh->getOmegaDotN(a, c, f);
            }
        }
        std::vector<UINT> deps(na * nc), blev(na * nc);
        for (UINT c = 0; c < nc; c++)
            for (UINT a = 0; a < na; a++)
                deps[a * nc + c] = g_graphTraverserForward->c_initNumDependencies(a, c);
        Mat2<UINT> prio(nc, na);
        Priorities::calcPriorities(prio);
        for (UINT c = 0; c < nc; c++)
            for (UINT a = 0; a < na; a++) blev[a * nc + c] = prio(c, a);
        dump_u64(pre + "adj.u64", adj);
        dump_u64(pre + "nbr.u64", nbr);
        dump_u64(pre + "f2c.u64", f2c);
        dump_u64(pre + "c2f.u64", c2f);
        dump_u64(pre + "deps.u64", deps);
        dump_u64(pre + "blev.u64", blev);
        dump_f64(pre + "vol.f64", vol.data(), vol.size());
        dump_f64(pre + "area.f64", area.data(), area.size());
        dump_f64(pre + "odn.f64", odn.data(), odn.size());
        return 0;
    }
    if (mode == "sweep" && argc == 8) {
        setup(argv[2], atoi(argv[3]), atoi(argv[4]));
        g_sigmaT = load_f64(argv[5], g_nCells);
        g_sigmaS.assign(g_nCells, 0.0);
        PsiData source, psi;
        std::vector<double> s = load_f64(argv[6], source.size());
        for (size_t i = 0; i < source.size(); i++) source[i] = s[i];
        SweeperTraverse sweeper;
        sweeper.sweep(psi, source, false);
        dump_f64(argv[7], &psi[0], psi.size());
        return 0;
    }
    if (mode == "sweep_local" && argc == 10) {
        setup(argv[2], atoi(argv[3]), atoi(argv[4]), false);
        g_sigmaT = load_f64(argv[5], g_nCells);
        g_sigmaS.assign(g_nCells, 0.0);
        PsiData source, psi;
        PsiBoundData psiBound;
        std::vector<double> s = load_f64(argv[6], source.size());
        for (size_t i = 0; i < source.size(); i++) source[i] = s[i];
        std::vector<double> b = load_f64(argv[7], psiBound.size());
        for (size_t i = 0; i < psiBound.size(); i++) psiBound[i] = b[i];
        psi.setToValue(0.0);
        Util::sweepLocal(psi, source, psiBound);
        dump_f64(argv[8], &psi[0], psi.size());
        const UINT nc = g_nCells, ns = g_tychoMesh->getNSides();
        std::vector<UINT> adj(nc * 4), rank(nc * 4), side(nc * 4), lg(ns);
        for (UINT c = 0; c < nc; c++)
            for (UINT f = 0; f < 4; f++) {
                adj[c * 4 + f] = g_tychoMesh->getAdjCell(c, f);
                rank[c * 4 + f] = g_tychoMesh->getAdjRank(c, f);
                side[c * 4 + f] = g_tychoMesh->getSide(c, f);
            }
        for (UINT i = 0; i < ns; i++) lg[i] = g_tychoMesh->getLGSide(i);
        std::string pre = argv[9];
        dump_u64(pre + "adj.u64", adj);
        dump_u64(pre + "rank.u64", rank);
        dump_u64(pre + "side.u64", side);
        dump_u64(pre + "lgside.u64", lg);
        return 0;
    }
    if (mode == "si" && argc == 11) {
        setup(argv[2], atoi(argv[3]), atoi(argv[4]));
        g_sigmaT = load_f64(argv[5], g_nCells);
        g_sigmaS = load_f64(argv[6], g_nCells);
        g_iterMax = atoi(argv[8]);
        g_errMax = atof(argv[9]);
        PsiData source, psi;
        std::vector<double> s = load_f64(argv[7], source.size());
        for (size_t i = 0; i < source.size(); i++) source[i] = s[i];
        SweeperTraverse sweeper;
        SourceIteration::fixedPoint(sweeper, psi, source);
        dump_f64(argv[10], &psi[0], psi.size());
        return 0;
    }
    if (mode == "levels" && argc == 5) {
        setup(argv[2], atoi(argv[3]), 1);
        const UINT na = g_nAngles, nc = g_nCells;
        std::vector<UINT> angles(na);
        for (UINT a = 0; a < na; a++) angles[a] = a;
        std::set<UINT> neighborProcs;
        calcNeighborProcs(neighborProcs);
        Mat3<bool> hasChild(na, nc, g_nFacePerCell), hasParent(na, nc, g_nFacePerCell);
        /* the reference's constructor leaves hasParent unset where
           calcDependencies writes nothing: start both from false */
        for (UINT a = 0; a < na; a++)
            for (UINT c = 0; c < nc; c++)
                for (UINT f = 0; f < g_nFacePerCell; f++) hasChild(a, c, f) = hasParent(a, c, f) = false;
        calcDependencies(angles, hasChild, hasParent);
        Mat2<UINT> cellLevels(na, nc), sideLevels(na, g_tychoMesh->getNSides());
        cellLevels.setAll(0);
        sideLevels.setAll(0);
        const UINT nlevels = calcLevels(cellLevels, sideLevels, hasChild, hasParent, neighborProcs, angles,
                                        na, g_maxCellsPerStep);
        std::vector<UINT> out(na * nc + 1);
        for (UINT a = 0; a < na; a++)
            for (UINT c = 0; c < nc; c++) out[a * nc + c] = cellLevels(a, c);
        out[na * nc] = nlevels;
        dump_u64(argv[4], out);
        return 0;
    }
    if (mode == "bench" && (argc == 9 || argc == 10)) {
        /* bench <pmesh> <snOrder> <nGroups> <sigmaT.f64> <qiso.f64> <steps> <warmup>:
           times the reference's own SweeperTraverse::sweep of an isotropic
           source (phi layout, copied to every angle as the reference's PsiData
           source) on all OpenMP threads; prints one line "REFBENCH <json>". */
        setup(argv[2], atoi(argv[3]), atoi(argv[4]));
        g_sigmaT = load_f64(argv[5], g_nCells);
        g_sigmaS.assign(g_nCells, 0.0);
        const int steps = atoi(argv[7]), warm = atoi(argv[8]);
        PsiData source, psi;
        std::vector<double> q = load_f64(argv[6], g_nCells * 4 * g_nGroups);
        for (UINT c = 0; c < g_nCells; c++)
            for (UINT a = 0; a < g_nAngles; a++)
                for (UINT v = 0; v < 4; v++)
                    for (UINT g = 0; g < g_nGroups; g++) source(g, v, a, c) = q[(c * 4 + v) * g_nGroups + g];
        SweeperTraverse sweeper;
        for (int i = 0; i < warm; i++) sweeper.sweep(psi, source, false);
        double tot = 0.0, best = 1e300;
        for (int i = 0; i < steps; i++) {
            double t0 = omp_get_wtime();
            sweeper.sweep(psi, source, false);
            double dt = omp_get_wtime() - t0;
            tot += dt;
            if (dt < best) best = dt;
        }
        double checksum = 0.0;
        uint64_t hash = 0;
        const uint64_t *words = reinterpret_cast<const uint64_t *>(&psi[0]);
        for (size_t i = 0; i < psi.size(); i++) {
            checksum += psi[i];
            hash += words[i] * (2 * (uint64_t)i + 1);
        }
        if (argc == 10) {
            PhiData phi;
            Util::psiToPhi(phi, psi);
            dump_f64(argv[9], &phi[0], phi.size());
        }
        printf("REFBENCH {\"seconds_per_sweep\": %.9g, \"best_seconds\": %.9g, \"threads\": %d, "
               "\"steps\": %d, \"checksum\": %.17g, \"psi_hash\": \"%016llx\", \"psi_words\": %zu}\n",
               tot / steps, best, (int)g_nThreads, steps, checksum, (unsigned long long)hash, psi.size());
        return 0;
    }
    fprintf(stderr, "ref_dump: bad arguments\n");
    return 2;
}
