"""Problem definitions (the reference's Problem namespace, src/Problem.cc)
and the benchmark workloads.

hat_source / hat_l2_error restate Problem::hatSource / hatL2Error
(src/Problem.cc:47-134) for meshes on [0,100]^3; diff_between_groups the
reference's group-consistency check (src/Util.cc:55-79).  The benchmark family
(`workload`) extends the reference's two-material problem with per-cell
lognormal sigma_t, a lower-triangular downscatter matrix and a box source,
all drawn from seeded generators; q is the angular source density, the
reference's convention (src/Problem.cc:73-75).
"""
import numpy as np

CUBE_SIZE = 100.0


def hat_source(mesh, quad, sigma_t, sigma_s, n_groups):
    """Problem::hatSource (src/Problem.cc:47-82), psi layout."""
    t = mesh.tables()
    xyz = t["coords"][t["cell_nodes"].astype(np.int64)] - CUBE_SIZE / 2.0  # (c, v, 3)
    x, y, z = xyz[..., 0][:, None, :], xyz[..., 1][:, None, :], xyz[..., 2][:, None, :]
    xi, eta, mu = quad.xi[None, :, None], quad.eta[None, :, None], quad.mu[None, :, None]
    r = np.sqrt(x * x + y * y + z * z)
    with np.errstate(divide="ignore", invalid="ignore"):
        val = (-x / (30.0 * r) * xi - y / (30.0 * r) * eta - z / (30.0 * r) * mu
               + (sigma_t - sigma_s)[:, None, None] * (1.0 - r / 30.0))
    val = np.where(r <= 30.0, val, 0.0)
    return np.ascontiguousarray(np.repeat(val[..., None], n_groups, axis=3))


def hat_l2_error(mesh, psi):
    """Problem::hatL2Error (src/Problem.cc:91-134)."""
    t = mesh.tables()
    xyz = (t["coords"][t["cell_nodes"].astype(np.int64)] - CUBE_SIZE / 2.0).mean(axis=1)
    c = np.sqrt((xyz ** 2).sum(axis=1))
    act = np.where(c <= 30.0, 1.0 - c / 30.0, 0.0)
    val = psi.mean(axis=2)  # (c, a, g)
    diff = val - act[:, None, None]
    return float(np.sqrt((diff ** 2).sum() / (val ** 2).sum()))


def diff_between_groups(psi):
    """Util::diffBetweenGroups (src/Util.cc:55-79): the largest |psi_g -
    psi_0| over groups g >= 1, cells, angles and vertices, relative to the
    largest |psi_0| (0 when every group carries the same psi, as the
    reference's within-group problems do).  psi: PsiData layout (c, a, 4, G)."""
    p = np.asarray(psi)
    p0 = p[..., 0]
    max_entry = float(np.abs(p0).max())
    max_diff = float(np.abs(p[..., 1:] - p0[..., None]).max()) if p.shape[-1] > 1 else 0.0
    return max_diff / max_entry


def downscatter_matrix(n_groups, ratio):
    """Lower-triangular g' -> g matrix, row g split equally over g' <= g so
    that each row sums to `ratio` (sigma_s = sigma_t * matrix)."""
    m = np.zeros((n_groups, n_groups))
    for g in range(n_groups):
        m[g, : g + 1] = ratio / (g + 1)
    return m


# The workloads the benchmark and the parity tests run.
WORKLOADS = {
    # 8^3 hexes x 6 = 3,072 tets, S4, G=1, sigma_t=1, sigma_s=0.5, q=1, SI to 1e-10.
    "kuhn8_s4_g1": dict(n=8, jitter=0.0, sn=4, groups=1, sigma="uniform", sigma_t=1.0,
                        ratio=0.5, scatter="within", source="all", method="si", tol=1e-10),
    # 32^3 x 6 = 196,608 tets, +-0.05h jitter, S8, G=8, lognormal(0,0.5) sigma_t,
    # downscatter rows 0.6 sigma_t, q=1 in the central 1/8, GMRES(20) to 1e-10.
    "kuhn32_s8_g8": dict(n=32, jitter=0.05, sn=8, groups=8, sigma="lognormal", lognormal_s=0.5,
                         ratio=0.6, scatter="down", source="box", method="gmres", tol=1e-10,
                         restart=20),
    # The 32^3 problem at 24^3 x 6 = 82,944 tets (psi 1.4 GB in FP32, over
    # ten times L2): the size for multi-pass profiler captures.
    "kuhn24_s8_g8": dict(n=24, jitter=0.05, sn=8, groups=8, sigma="lognormal", lognormal_s=0.5,
                         ratio=0.6, scatter="down", source="box", method="gmres", tol=1e-10,
                         restart=20),
    # 64^3 x 6 = 1,572,864 tets, S8, G=16, lognormal(0,1), ratio 0.99, GMRES(30).
    "kuhn64_s8_g16": dict(n=64, jitter=0.05, sn=8, groups=16, sigma="lognormal", lognormal_s=1.0,
                          ratio=0.99, scatter="down", source="box", method="mixed", tol=1e-10,
                          restart=30),
}


def make_problem(n, jitter, sn, groups, sigma="uniform", sigma_t=1.0, lognormal_s=0.5,
                 ratio=0.5, scatter="within", source="all", seed=1234, length=1.0, **_):
    """Builds (mesh, sigma_t, sigma_s, scatter_matrix or None, q_iso)."""
    from .sweeper import TychoMesh
    mesh = TychoMesh.kuhn_cube(n, jitter, seed, length)
    rng = np.random.default_rng(seed + 1)
    nc = mesh.n_cells
    if sigma == "uniform":
        st = np.full(nc, float(sigma_t))
    else:
        st = np.exp(rng.normal(0.0, lognormal_s, nc))
    if scatter == "within":
        ss = ratio * st
        mat = None
    else:
        ss = st.copy()
        mat = downscatter_matrix(groups, ratio)
    q = np.zeros((nc, 4, groups))
    if source == "all":
        q[:] = 1.0
    else:
        cen = mesh.centroids() / length
        inside = np.all((cen >= 0.25) & (cen <= 0.75), axis=1)
        q[inside] = 1.0
    return mesh, st, ss, mat, q


def batch_instances(count=256, seed=4321, n_range=(4, 24), groups=(1, 2, 4, 8), sn_orders=(4, 6, 8),
                    ratio_range=(0.3, 0.95), lognormal_s=0.5, jitter=0.05):
    """Parameters of `count` independent uneven problems: n ~ U{n_range},
    G ~ U{groups}, S ~ U{sn_orders}, sigma_t ~ lognormal(0, lognormal_s) per
    cell, scattering ratio c ~ U[ratio_range] (downscatter rows summing to c
    for G > 1, within-group for G = 1), isotropic q = 1 everywhere, interior
    vertices jittered by +-jitter*h -- all seeded.  Returns a list of dicts
    for make_problem (each with its own seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        G = int(rng.choice(groups))
        out.append(dict(n=int(rng.integers(n_range[0], n_range[1] + 1)), jitter=jitter,
                        sn=int(rng.choice(sn_orders)), groups=G, sigma="lognormal",
                        lognormal_s=lognormal_s, ratio=float(rng.uniform(*ratio_range)),
                        scatter="within" if G == 1 else "down", source="all",
                        seed=int(seed * 1000 + k)))
    return out


def footprint_bytes(n_cells, n_angles, groups, fp32=True, records=True):
    """Device memory of one resident instance (tycho::Sweeper plus its batch
    vectors): psi (FP64-sized, shared by the FP32 sweep), per-item face terms,
    schedule, completion flags and records, per-cell tables, phi-sized
    vectors."""
    items = n_cells * n_angles  # padding to 32 per level adds a little
    phi = n_cells * 4 * groups * 8
    b = items * 4 * groups * 8            # psi
    b += items * (32 + (16 if fp32 else 0))  # item face terms
    b += items * (4 + 4)                  # item list, completion flags
    if records:
        b += items * (256 + (128 if fp32 else 0))
    b += n_cells * (16 + 4 + 24 + 12 + 8 + 8)  # adjacency, maps, cell terms, sigma
    b += phi * (6 + (3 if fp32 else 0))   # phi, iso, r, tmp (+ FP32 iso, batch r/d/k)
    return int(b * 1.03)
