"""`python -m tycho2_b200.run <pmesh> <deck>`: the reference's command line
on the B200 sweep, on the reference's own regression problem (cube-208, the
gold deck).  One partition: SourceIteration true and false reproduce
test/regression/gold.psi within diff.py's 1e-10 (relative L1 and Linf) and
print the reference's hatL2Error of it; two partitions (the reference's
PartitionColumns 2 1): the PBJ and Schur sweep types reach gold within 1e-8."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from helpers import gold_psi
from test_run_cli import GOLD_DECK

pytestmark = pytest.mark.gpu

PARTITION_COLUMNS = os.path.join(ROOT, "oracle", "_ref", "PartitionColumns.x")


def _rel(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum()), float(np.abs(a - b).max() / np.abs(b).max())


def _deck(d, name, **changes):
    text = GOLD_DECK.replace("OutputFilename  out.psi", "OutputFilename  " + os.path.join(d, name + ".psi"))
    for k, v in changes.items():
        lines = [ln for ln in text.splitlines() if not ln.lower().startswith(k.lower() + " ")]
        text = "\n".join(lines + ["%s %s" % (k, v)]) + "\n"
    path = os.path.join(d, name + ".deck")
    with open(path, "w") as f:
        f.write(text)
    return path


@pytest.mark.parametrize("si", [True, False])
def test_gold_deck_one_partition(built, workdir, si):
    import io
    import tycho2_b200 as ty
    from tycho2_b200 import problems
    from tycho2_b200.run import run
    d = str(workdir)
    pm = os.path.join(d, "cube208_run.pmesh")
    mesh = ty.TychoMesh.read_smesh(os.path.join(GOLDEN, "cube-208.smesh"))
    mesh.write_pmesh(pm)
    name = "gold_si" if si else "gold_krylov"
    out = io.StringIO()
    res = run(pm, _deck(d, name, SourceIteration="true" if si else "false"), out=out)
    raw = np.fromfile(os.path.join(d, name + ".psi"))
    psi = raw[8:].reshape(208, 128, 4, 2)
    l1, linf = _rel(psi, gold_psi())
    assert l1 <= 1e-10 and linf <= 1e-10, (l1, linf)
    if si:
        assert res["iterations"] == 34
    want = problems.hat_l2_error(mesh, gold_psi())
    assert abs(res["l2_error"] - want) <= 1e-8 * want
    assert res["diff_between_groups"] == 0.0
    assert "L2 Relative Error:" in out.getvalue() and "Diff between groups:" in out.getvalue()


@pytest.mark.skipif(not os.path.exists(PARTITION_COLUMNS), reason="reference's PartitionColumns not built")
@pytest.mark.parametrize("sweep_type", ["PBJSI", "PBJ", "Schur", "SchurKrylov"])
def test_gold_deck_two_partitions(built, workdir, sweep_type):
    import io
    from tycho2_b200.run import run
    d = str(workdir)
    pm = os.path.join(d, "cube208_p2.pmesh")
    if not os.path.exists(pm):
        subprocess.run([PARTITION_COLUMNS, "2", "1", os.path.join(GOLDEN, "cube-208.smesh"), pm], check=True,
                       stdout=subprocess.DEVNULL)
    name = "gold_p2_" + sweep_type
    res = run(pm, _deck(d, name, SweepType=sweep_type, DD_ErrMax="1e-12"), out=io.StringIO())
    assert res["partitions"] == 2
    psi = np.fromfile(os.path.join(d, name + ".psi"))[8:].reshape(208, 128, 4, 2)
    l1, linf = _rel(psi, gold_psi())
    assert l1 <= 1e-8 and linf <= 1e-8, (sweep_type, l1, linf)


@pytest.mark.skipif(not os.path.exists(PARTITION_COLUMNS), reason="reference's PartitionColumns not built")
def test_pipelined_traversal_is_refused_on_partitions(built, workdir):
    from tycho2_b200.run import run
    d = str(workdir)
    pm = os.path.join(d, "cube208_p2.pmesh")
    if not os.path.exists(pm):
        subprocess.run([PARTITION_COLUMNS, "2", "1", os.path.join(GOLDEN, "cube-208.smesh"), pm], check=True,
                       stdout=subprocess.DEVNULL)
    with pytest.raises(ValueError, match="pipelined"):
        run(pm, _deck(d, "refused", SweepType="TraverseGraph"))


@pytest.mark.skipif(not os.path.exists(PARTITION_COLUMNS), reason="reference's PartitionColumns not built")
@pytest.mark.timeout(600)
def test_two_ranks_under_torchrun(built, workdir):
    """torchrun with two ranks, one partition each (gloo, both on this GPU:
    their sweeps never wait on each other): the PBJSI deck writes the same
    .psi as all partitions in one process."""
    import io
    import sys
    from tycho2_b200.run import run
    d = str(workdir)
    pm = os.path.join(d, "cube208_p2.pmesh")
    if not os.path.exists(pm):
        subprocess.run([PARTITION_COLUMNS, "2", "1", os.path.join(GOLDEN, "cube-208.smesh"), pm], check=True,
                       stdout=subprocess.DEVNULL)
    run(pm, _deck(d, "one_proc", SweepType="PBJSI"), out=io.StringIO())
    deck = _deck(d, "two_ranks", SweepType="PBJSI")
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    r = subprocess.run(["timeout", "-k", "30", "500", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                        "--nproc-per-node", "2", "--master-addr", "127.0.0.1", "--master-port", str(port),
                        "-m", "tycho2_b200.run", pm, deck, "--backend", "gloo"],
                       cwd=ROOT, capture_output=True, text=True, timeout=560)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-3000:]
    assert "L2 Relative Error:" in r.stdout
    a = np.fromfile(os.path.join(d, "one_proc.psi"))
    b = np.fromfile(os.path.join(d, "two_ranks.psi"))
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
