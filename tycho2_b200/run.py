"""The reference's command line on the B200 sweep.

    python -m tycho2_b200.run <parallel mesh> <input deck>

reads what the reference's `sweep.x <parallel mesh> <input deck>` reads --
the deck keys of src/Main.cc:97-184 (KeyValueReader format: one `key value`
per line, `#` comments, keys compared without case) -- builds the
reference's problem (Problem::createCrossSections: material 1 / 2 cross
sections, src/Problem.cc:149-172; Problem::getSource: the hat source,
:140-143), solves it, writes the .psi file (PsiData::writeToFile format)
when OutputFile is true, and prints the reference's closing checks
(src/Main.cc:340-344: Problem::hatL2Error, Util::diffBetweenGroups).

SweepType on a one-partition mesh: every type solves the whole mesh on one
GPU (TraverseGraph, OriginalTycho1/2; the PBJ and Schur types reduce to it
with one partition); intraAngleP picks the work order within a wavefront
(0 random, 1 b-levels, otherwise cell order; psi is the same).  On a
multi-partition mesh: PBJ, PBJOuter, PBJSI, Schur, SchurOuter, SchurKrylov
(tycho2_b200.partitions), one partition per rank under torch.distributed
(torchrun, NCCL) or all partitions in this process, spread over the
visible GPUs; the pipelined multi-rank TraverseGraph / OriginalTycho sweeps
are not available there.  SourceIteration true: source iteration to
errMax, false: GMRES(30) (the reference's PETSc default restart).
"""
import argparse
import os
import re
import sys

import numpy as np

from . import partitions, problems
from .sweeper import Quadrature, SweeperCuda, TychoMesh

_BOOL = {"true": True, "false": False}


def read_deck(path):
    """KeyValueReader (src/KeyValueReader.cc): key -> value strings, keys
    lower-cased; `#` starts a comment.  Values may also hold characters the
    reference's tokens do not (a path for OutputFilename)."""
    deck = {}
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0].strip()
            if not line:
                continue
            m = re.match(r"([A-Za-z0-9+\-_.]+)\s+(\S+)", line)
            if not m:
                raise ValueError("cannot parse deck line: %r" % line)
            deck[m.group(1).lower()] = m.group(2)
    return deck


def _get(deck, key, kind, default=None):
    v = deck.get(key.lower())
    if v is None:
        if default is None:
            raise KeyError("deck key %s missing" % key)
        v = str(default)
    if kind is bool:
        if v.lower() not in _BOOL:
            raise ValueError("deck key %s: %s is not true/false" % (key, v))
        return _BOOL[v.lower()]
    return kind(v)


def cross_sections(mesh, sigma_t1, sigma_s1, sigma_t2, sigma_s2):
    """Problem::createCrossSections: per cell by material index 1 or 2."""
    mat = mesh.cell_material()
    if np.any((mat != 1) & (mat != 2)):
        raise ValueError("Material index out of bounds.")
    st = np.where(mat == 1, sigma_t1, sigma_t2).astype(np.float64)
    ss = np.where(mat == 1, sigma_s1, sigma_s2).astype(np.float64)
    return st, ss


def write_psi(path, parts_psi, n_cells_global, n_angles, n_groups):
    """PsiData::writeToFile (src/PsiData.cc:62-106): 32-byte name, version,
    cells, angles, groups, then each cell's psi at its global position.
    parts_psi: (cell_gid, psi (c, A, 4, G)) per partition."""
    per = n_angles * 4 * n_groups
    out = np.zeros((n_cells_global, per))
    for gid, psi in parts_psi:
        out[gid.astype(np.int64)] = psi.reshape(psi.shape[0], per)
    name = b"Tycho 2 Psi Output".ljust(32, b"\0")
    with open(path, "wb") as f:
        f.write(name)
        f.write(np.array([1, n_cells_global, n_angles, n_groups], np.uint64).tobytes())
        f.write(out.tobytes())


def _hat_sums(mesh, psi):
    """Problem::hatL2Error's two sums over one partition's cells."""
    t = mesh.tables()
    xyz = (t["coords"][t["cell_nodes"].astype(np.int64)] - problems.CUBE_SIZE / 2.0).mean(axis=1)
    c = np.sqrt((xyz ** 2).sum(axis=1))
    act = np.where(c <= 30.0, 1.0 - c / 30.0, 0.0)
    val = psi.mean(axis=2)
    return float(((val - act[:, None, None]) ** 2).sum()), float((val ** 2).sum())


def _group_sums(psi):
    p0 = psi[..., 0]
    d = float(np.abs(psi[..., 1:] - p0[..., None]).max()) if psi.shape[-1] > 1 else 0.0
    return d, float(np.abs(p0).max())


def run(pmesh, deck_path, devices=None, out=sys.stdout):
    """Runs one deck; returns a dict of what it printed and the iteration
    counts."""
    deck = read_deck(deck_path)
    sn = _get(deck, "snOrder", int)
    groups = _get(deck, "nGroups", int)
    iter_max = _get(deck, "iterMax", int)
    err_max = _get(deck, "errMax", float)
    st1, ss1 = _get(deck, "sigmaT1", float), _get(deck, "sigmaS1", float)
    st2, ss2 = _get(deck, "sigmaT2", float), _get(deck, "sigmaS2", float)
    use_si = _get(deck, "SourceIteration", bool)
    sweep_type = _get(deck, "SweepType", str)
    gauss = _get(deck, "GaussElim", str, "NoPivot")
    output = _get(deck, "OutputFile", bool, "false")
    output_name = _get(deck, "OutputFilename", str, "out.psi")
    dd_iter_max = _get(deck, "DD_IterMax", int, "100")
    dd_err_max = _get(deck, "DD_ErrMax", float, "1e-10")
    intra = _get(deck, "intraAngleP", int, "3")
    method = "si" if use_si else "krylov"

    import torch.distributed as dist
    distributed = dist.is_available() and dist.is_initialized()
    head = TychoMesh.read_pmesh(pmesh, dist.get_rank() if distributed else 0)
    P = head.n_partitions
    quad = Quadrature(sn)
    result = {"sweep_type": sweep_type, "partitions": P}

    if P == 1:
        sw = SweeperCuda(head, sn, groups, gauss_elim=gauss, device=(devices or [0])[0])
        st, ss = cross_sections(head, st1, ss1, st2, ss2)
        sw.set_cross_sections(st, ss)
        sw.set_source(problems.hat_source(head, quad, st, ss, groups), "angular")
        sw.set_work_order({0: "random", 1: "blevel"}.get(intra, "cell"))
        phi, psi, stats = sw.solve("si" if use_si else "gmres", iter_max=iter_max, err_max=err_max,
                                   restart=30)
        result["iterations"] = stats["iterations"]
        parts_psi = [(head.tables()["cell_gid"], psi)]
        meshes = [head]
        sw.close()
    else:
        solvers = {"pbj": lambda ps: partitions.pbj(ps, iter_max, err_max, dd_iter_max, dd_err_max, method),
                   "pbjouter": lambda ps: partitions.pbj_outer(ps, iter_max, err_max, dd_iter_max,
                                                               dd_err_max, method),
                   "pbjsi": lambda ps: partitions.pbj_si(ps, dd_iter_max, dd_err_max),
                   "schur": lambda ps: partitions.schur(ps, iter_max, err_max, dd_iter_max, dd_err_max,
                                                        method),
                   "schurouter": lambda ps: partitions.schur_outer(ps, iter_max, err_max, dd_iter_max,
                                                                   dd_err_max),
                   "schurkrylov": lambda ps: partitions.schur_krylov(ps, dd_iter_max, dd_err_max)}
        key = sweep_type.lower()
        if key not in solvers:
            raise ValueError("SweepType %s on a %d-partition mesh: the pipelined multi-rank traversal is not "
                             "available; use PBJ, PBJOuter, PBJSI, Schur, SchurOuter or SchurKrylov"
                             % (sweep_type, P))
        if distributed:
            if dist.get_world_size() != P:
                raise ValueError("%d partitions need %d ranks" % (P, P))
            import torch
            mine = [dist.get_rank()]
            devs = [torch.cuda.current_device()]
        else:
            import torch
            mine = list(range(P))
            devs = devices or list(range(max(1, torch.cuda.device_count())))
        parts, meshes = [], []
        for i, p in enumerate(mine):
            mesh = head if p == head.partition else TychoMesh.read_pmesh(pmesh, p)
            sw = SweeperCuda(mesh, sn, groups, gauss_elim=gauss, device=devs[i % len(devs)])
            st, ss = cross_sections(mesh, st1, ss1, st2, ss2)
            sw.set_cross_sections(st, ss)
            sw.set_source(problems.hat_source(mesh, quad, st, ss, groups), "angular")
            parts.append(partitions.GpuPartition(sw))
            meshes.append(mesh)
        ps = partitions.DistributedPartitions(parts[0]) if distributed else partitions.PartitionSet(parts)
        r = solvers[key](ps)
        result["iterations"] = r[1]
        parts_psi = [(p.gid, p.sw.read_psi()) for p in parts]
        for p in parts:
            p.sw.close()

    # the closing checks, summed over the partitions (Comm::gsum / gmax)
    hs = np.array([_hat_sums(m, psi) for m, (_, psi) in zip(meshes, parts_psi)]).sum(axis=0)
    gs = [_group_sums(psi) for _, psi in parts_psi]
    sums = [hs[0], hs[1], max(g[0] for g in gs), max(g[1] for g in gs)]
    if P > 1 and distributed:
        import torch
        t = torch.tensor(sums[:2], dtype=torch.float64)
        m = torch.tensor(sums[2:], dtype=torch.float64)
        if dist.get_backend() == "nccl":
            t, m = t.cuda(), m.cuda()
        dist.all_reduce(t)
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
        sums = t.cpu().tolist() + m.cpu().tolist()
    l2 = float(np.sqrt(sums[0] / sums[1]))
    diff = sums[2] / sums[3]
    result.update(l2_error=l2, diff_between_groups=diff)
    rank0 = not distributed or dist.get_rank() == 0
    if output:
        if distributed and P > 1:
            gathered = [None] * dist.get_world_size()
            dist.all_gather_object(gathered, parts_psi)
            parts_psi = [x for g in gathered for x in g]
        if rank0:
            n_global = int(sum(psi.shape[0] for _, psi in parts_psi))
            write_psi(output_name, parts_psi, n_global, quad.n_angles, groups)
            result["output"] = output_name
    if rank0:
        print("L2 Relative Error: %e" % l2, file=out)
        print("Diff between groups: %e" % diff, file=out)
    return result


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("pmesh")
    ap.add_argument("deck")
    ap.add_argument("--devices", default=None, help="comma-separated CUDA devices for the partitions "
                                                     "of one process (default: all visible)")
    ap.add_argument("--backend", default="nccl", choices=["nccl", "gloo"],
                    help="torch.distributed backend under torchrun (gloo: packets through host memory)")
    a = ap.parse_args(argv)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")) % max(1, torch.cuda.device_count()))
        dist.init_process_group(a.backend, timeout=datetime.timedelta(seconds=300))
    devs = [int(x) for x in a.devices.split(",")] if a.devices else None
    try:
        res = run(a.pmesh, a.deck, devs)
    finally:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()
    return res


if __name__ == "__main__":
    main()
