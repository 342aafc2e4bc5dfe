/*
 * SweeperCuda.hh -- the reference-side adapter: a tycho2 SweeperAbstract
 * (src/SweeperAbstract.hh:47-70) whose sweep runs on a B200 through the C ABI
 * in include/tycho_cuda.h.  Header-only; a maintainer adds it next to the
 * reference's sweepers, adds `SweepType_Cuda` to src/Global.hh:86-97, a
 * "Cuda" branch to the SweepType parser (src/Main.cc:143-164) and a
 * `case SweepType_Cuda: sweeper = new SweeperCuda(); break;` to the sweeper
 * switch (src/Main.cc:269-321), and links libtycho_b200.so.
 *
 *   sweep(psi, source)  == SweeperTraverse::sweep (src/SweeperTraverse.cc:82-89):
 *                          psi = L^{-1} source on the GPU; SourceIteration's
 *                          host loops (fixedPoint, krylov, lhsOperator) call it
 *                          unchanged.
 *   solve()             == SweeperTraverse::solve (src/SweeperTraverse.cc:65-74):
 *                          same problem and stopping rules (deck keys iterMax,
 *                          errMax, SourceIteration), with the outer iteration
 *                          resident on the device; psi lands in c_psi.
 *   sweepLocal(psi, source, psiBound)
 *                       == Util::sweepLocal (src/Util.cc:138-145) on one MPI
 *                          rank's partition: the PBJ and Schur sweepers'
 *                          local sweep (src/SweeperPBJ.cc, src/SweeperSchur.cc),
 *                          with psiBound on the faces toward other ranks.
 *
 * The mesh comes from g_tychoMesh's own tables (no second file read), the
 * quadrature from g_snOrder, cross sections from g_sigmaT / g_sigmaS.  A
 * nonzero status is reported through Insist, as the reference reports its
 * own failures (src/Assert.hh:62).
 *
 * The sweeper's own psi and source (c_psi, c_source: host `new double[]`,
 * src/PsiData.hh:94-103) are page-locked for its lifetime, so a sweep that
 * receives c_psi -- SweeperTraverse::solve hands it to fixedPoint and
 * krylov (src/SweeperTraverse.cc:65-74) -- copies it back asynchronously,
 * in angle chunks that overlap the other direction's copies and the sweep.
 * Buffers the adapter does not own (fixedPoint's local totalSource) stay
 * pageable: the adapter cannot know when they are freed.
 */
#ifndef __SWEEPER_CUDA_HH__
#define __SWEEPER_CUDA_HH__

#include <string>
#include <vector>

#include "Assert.hh"
#include "Comm.hh"
#include "Global.hh"
#include "Problem.hh"
#include "PsiData.hh"
#include "SweeperAbstract.hh"
#include "TychoMesh.hh"
#include "tycho_cuda.h"

class SweeperCuda : public SweeperAbstract
{
public:
    SweeperCuda()
    : c_mesh(NULL), c_sweeper(NULL)
    {
        c_locked[0] = c_locked[1] = false;
        const UINT nc = g_nCells, nn = g_tychoMesh->getNNodes();
        std::vector<uint64_t> cellNodes(nc * 4), adj(nc * 4), f2c(nc * 12), gid(nc);
        std::vector<double> coords(nn * 3);
        for (UINT n = 0; n < nn; n++)
            for (UINT d = 0; d < 3; d++) coords[n * 3 + d] = g_tychoMesh->getNodeCoord(n, d);
        for (UINT c = 0; c < nc; c++) {
            gid[c] = g_tychoMesh->getLGCell(c);
            for (UINT f = 0; f < 4; f++) {
                cellNodes[c * 4 + f] = g_tychoMesh->getCellNode(c, f);
                adj[c * 4 + f] = g_tychoMesh->getAdjCell(c, f);
                for (UINT k = 0; k < 3; k++)
                    f2c[(c * 4 + f) * 3 + k] = g_tychoMesh->getFaceToCellVrtx(c, f, k);
            }
        }
        check(tycho_mesh_from_arrays(nc, nn, cellNodes.data(), coords.data(), adj.data(),
                                     f2c.data(), gid.data(), &c_mesh));
        // this rank's partition: the faces toward other ranks read psiBound
        // in sweepLocal (src/TychoMeshIO.cc:228-262)
        if (Comm::numRanks() > 1) {
            const UINT ns = g_tychoMesh->getNSides();
            std::vector<uint64_t> rank(nc * 4), lgside(ns);
            for (UINT c = 0; c < nc; c++)
                for (UINT f = 0; f < 4; f++) rank[c * 4 + f] = g_tychoMesh->getAdjRank(c, f);
            for (UINT s = 0; s < ns; s++) lgside[s] = g_tychoMesh->getLGSide(s);
            check(tycho_mesh_set_partition(c_mesh, (uint64_t)Comm::rank(), (uint64_t)Comm::numRanks(),
                                           rank.data(), lgside.data()));
        }
        tycho_sweeper_opts opts = {};
        opts.sn_order = (int)g_snOrder;
        opts.n_groups = (int)g_nGroups;
        opts.gauss_elim = g_gaussElim == GaussElim_Original     ? TYCHO_GAUSS_ORIGINAL
                          : g_gaussElim == GaussElim_CramerGlu   ? TYCHO_GAUSS_CRAMER_GLU
                          : g_gaussElim == GaussElim_CramerIntel ? TYCHO_GAUSS_CRAMER_INTEL
                                                                 : TYCHO_GAUSS_NOPIVOT;
        opts.device = 0;
        opts.fp32 = 0;
        opts.tpi64 = 0;
        opts.tpi32 = 0;
        opts.schedule = 0;
        check(tycho_sweeper_create(c_mesh, &opts, &c_sweeper));
        check(tycho_sweeper_set_cross_sections(c_sweeper, g_sigmaT.data(), g_sigmaS.data(), NULL));
        // page-locked if the system allows it; pageable otherwise
        c_locked[0] = tycho_host_register(&c_psi[0], c_psi.size() * sizeof(double)) == TYCHO_OK;
        c_locked[1] = tycho_host_register(&c_source[0], c_source.size() * sizeof(double)) == TYCHO_OK;
    }

    ~SweeperCuda()
    {
        if (c_locked[0]) tycho_host_unregister(&c_psi[0]);
        if (c_locked[1]) tycho_host_unregister(&c_source[0]);
        tycho_sweeper_destroy(c_sweeper);
        tycho_mesh_free(c_mesh);
    }

    void sweep(PsiData &psi, const PsiData &source, bool zeroPsiBound = false)
    {
        UNUSED_VARIABLE(zeroPsiBound);  // psiBound as last set (none: vacuum)
        check(tycho_sweeper_sweep(c_sweeper, &source[0], &psi[0]));
    }

    // Util::sweepLocal(psi, source, psiBound) (src/Util.cc:138-145) on the
    // GPU: this rank's partition swept with the incoming psi on faces toward
    // other ranks taken from psiBound, as the PBJ and Schur sweepers call it
    // (src/SweeperPBJ.cc:129-138, :179, :287).
    void sweepLocal(PsiData &psi, const PsiData &source, const PsiBoundData &psiBound)
    {
        check(tycho_sweeper_set_psi_bound(c_sweeper, &psiBound[0]));
        check(tycho_sweeper_sweep(c_sweeper, &source[0], &psi[0]));
    }

    void solve()
    {
        Problem::getSource(c_source);
        c_psi.setToValue(0.0);
        check(tycho_sweeper_set_source(c_sweeper, 0, &c_source[0]));
        tycho_solve_opts o;
        o.method = g_useSourceIteration ? TYCHO_SOURCE_ITERATION : TYCHO_GMRES;
        o.iter_max = (int)g_iterMax;
        o.err_max = g_errMax;
        o.restart = 30;
        o.inner_tol = 0.0;
        o.refine_max = 0;
        tycho_solve_stats st;
        check(tycho_sweeper_solve(c_sweeper, &o, NULL, &c_psi[0], &st));
        printf("SweeperCuda: %d iterations, error %e, %.3f s on the device\n",
               st.iterations, st.final_error, st.seconds);
    }

private:
    static void check(int status)
    {
        if (status != TYCHO_OK) {
            char msg[512];
            tycho_last_error(msg, sizeof msg);
            Insist(false, msg);
        }
    }

    tycho_mesh *c_mesh;
    tycho_sweeper *c_sweeper;
    bool c_locked[2];
};

#endif
