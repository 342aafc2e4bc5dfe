/*
 * tycho_oracle.c -- CPU restatement of lanl/tycho2's linear-discontinuous SN
 * sweep path.  TEST INFRASTRUCTURE ONLY: this file is the checker that the
 * B200 sweep is compared against.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it; the product never links it.
 *
 * Parity is pinned two ways (see tests/test_oracle_*.py):
 *   - against the reference's own golden vector test/regression/gold.psi
 *     (cube-208, S8, G=2, sigma_t=10, sigma_s=5, hat source, SI to 1e-10);
 *   - against the reference itself, compiled from its sources under
 *     oracle/_ref (oracle/Makefile), on meshes written by this project.
 *
 * Everything is double precision and written with the reference's operation
 * order, so that results are bit-identical to the reference's build (compile
 * with -ffp-contract=off).  Each function cites the reference file:line that
 * it restates; all paths are relative to the tycho2 source tree.
 *
 * Layouts follow the reference containers:
 *   psi / angular source : ((c*A + a)*4 + v)*G + g      (src/PsiData.hh:155-163)
 *   phi / isotropic src  : (c*4 + v)*G + g              (src/PsiData.hh:363-370)
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../tycho2_b200/csrc/gauss_legendre_tables.h"

#define OR_NONE UINT64_MAX
#define OR_PI 3.14159265358979323846

/* ------------------------------------------------------------------------ */
/* Mesh (src/ParallelMesh.hh:43-81 file format, src/TychoMeshIO.cc:153-333) */
/* ------------------------------------------------------------------------ */

typedef struct {
    uint64_t nc, nn, nf, nsides;
    double *coords;          /* (node,3) */
    uint64_t *cell_nodes;    /* (c,4) */
    uint64_t *cell_faces;    /* (c,4) bounding faces, file order */
    uint64_t *face_cells;    /* (face,2) */
    uint64_t *face_nodes;    /* (face,3) */
    uint64_t *face_btype;    /* face boundary type */
    uint64_t *face_gid;      /* face global id */
    uint64_t *face_part;     /* (face,2) partitions of its two sides */
    uint64_t *cell_gid, *cell_mat;
    uint64_t part, nparts;   /* which partition of how many */
    uint64_t *adj_rank;      /* (c,f) partition across the face, OR_NONE on the mesh boundary */
    uint64_t *side_gid;      /* (side) global face id of each side */
    /* TychoMesh tables */
    uint64_t *adj_cell;      /* (c,f) */
    uint64_t *adj_face;      /* (c,f) */
    uint64_t *side;          /* (c,f) */
    uint64_t *f2c;           /* (c,f,fv) faceToCellVrtx */
    uint64_t *c2f;           /* (c,f,cv) cellToFaceVrtx, OR_NONE on cv == f */
    uint64_t *nbr_vrtx;      /* (c,f,fv) neighborVrtx */
    double *volume;          /* c */
    double *area;            /* (c,f) */
    double *normal;          /* (c,f,3) outward unit normals */
} OMesh;

static int read_u64(FILE *fp, uint64_t *dst, size_t n)
{
    return fread(dst, sizeof(uint64_t), n, fp) == n ? 0 : -1;
}

/* getLFaceIndex: face k of a cell is the face opposite cell vertex k
   (src/TychoMeshIO.cc:128-145). */
static uint64_t lface_index(const uint64_t cn[4], const uint64_t fn[3])
{
    for (uint64_t v = 0; v < 4; v++)
        if (cn[v] != fn[0] && cn[v] != fn[1] && cn[v] != fn[2]) return v;
    return OR_NONE;
}

/* Triangle area 1/2|AxB| (src/TychoMesh.cc:67-86). */
static double tri_area(const double p[3][3])
{
    double a[3], b[3], c[3];
    for (int d = 0; d < 3; d++) { a[d] = p[1][d] - p[0][d]; b[d] = p[2][d] - p[0][d]; }
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
    return 0.5 * sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
}

/* Tet volume 1/6|C.(AxB)| (src/TychoMesh.cc:95-117). */
static double tet_volume(const double p[4][3])
{
    double a[3], b[3], c[3], x[3];
    for (int d = 0; d < 3; d++) {
        a[d] = p[1][d] - p[0][d]; b[d] = p[2][d] - p[0][d]; c[d] = p[3][d] - p[0][d];
    }
    x[0] = a[1] * b[2] - a[2] * b[1];
    x[1] = a[2] * b[0] - a[0] * b[2];
    x[2] = a[0] * b[1] - a[1] * b[0];
    return 1.0 / 6.0 * fabs(x[0] * c[0] + x[1] * c[1] + x[2] * c[2]);
}

/* Outward unit normal of a face (src/TychoMesh.cc:124-187). */
static void face_normal(const double fp[3][3], const double cp[4][3], double n[3])
{
    double a[3], b[3], c[3];
    for (int d = 0; d < 3; d++) { a[d] = fp[1][d] - fp[0][d]; b[d] = fp[2][d] - fp[0][d]; }
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
    double norm = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    n[0] = c[0] / norm; n[1] = c[1] / norm; n[2] = c[2] / norm;
    int vi;
    for (vi = 0; vi < 4; vi++) {
        int eq = 0;
        for (int k = 0; k < 3; k++)
            if (cp[vi][0] == fp[k][0] && cp[vi][1] == fp[k][1] && cp[vi][2] == fp[k][2]) eq = 1;
        if (!eq) break;
    }
    if (vi == 4) vi = 3; /* degenerate: the reference reads past the loop */
    double dot = n[0] * (cp[vi][0] - fp[0][0]) + n[1] * (cp[vi][1] - fp[0][1]) +
                 n[2] * (cp[vi][2] - fp[0][2]);
    if (dot > 0) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
}

void om_free(OMesh *m)
{
    if (!m) return;
    free(m->coords); free(m->cell_nodes); free(m->cell_faces); free(m->face_cells);
    free(m->face_nodes); free(m->face_btype); free(m->cell_gid); free(m->cell_mat);
    free(m->face_gid); free(m->face_part); free(m->adj_rank); free(m->side_gid);
    free(m->adj_cell); free(m->adj_face); free(m->side); free(m->f2c); free(m->c2f);
    free(m->nbr_vrtx); free(m->volume); free(m->area); free(m->normal);
    free(m);
}

/* Reads partition `part` of a .pmesh (part < 0: the file must hold one
   partition) and builds the TychoMesh tables of that MPI rank's view
   (src/ParallelMesh.cc:581-690, src/TychoMeshIO.cc:153-333).  Returns NULL
   on any format error. */
OMesh *om_load_pmesh_part(const char *path, int64_t part)
{
    static const char name[32] = "Tycho 2 Parallel Mesh";
    FILE *fp = fopen(path, "rb");
    if (!fp) return NULL;
    OMesh *m = (OMesh *)calloc(1, sizeof(OMesh));
    char hdr[32];
    uint64_t vp[2], off, cnt[3];
    if (fread(hdr, 1, 32, fp) != 32 || memcmp(hdr, name, 32) != 0) goto fail;
    if (read_u64(fp, vp, 2) || vp[0] != 2 || vp[1] == 0) goto fail;
    if (part < 0 && vp[1] != 1) goto fail;
    if (part < 0) part = 0;
    if ((uint64_t)part >= vp[1]) goto fail;
    m->part = (uint64_t)part;
    m->nparts = vp[1];
    if (fseek(fp, (long)(32 + (2 + part) * 8), SEEK_SET) != 0 || read_u64(fp, &off, 1)) goto fail;
    if (fseek(fp, (long)off, SEEK_SET) != 0) goto fail;
    if (read_u64(fp, cnt, 3)) goto fail;
    m->nc = cnt[0]; m->nf = cnt[1]; m->nn = cnt[2];
    {
        uint64_t *cbuf = (uint64_t *)malloc(sizeof(uint64_t) * m->nc * 10);
        uint64_t *fbuf = (uint64_t *)malloc(sizeof(uint64_t) * m->nf * 9);
        uint64_t *nbuf = (uint64_t *)malloc(sizeof(uint64_t) * m->nn * 4);
        int bad = read_u64(fp, cbuf, m->nc * 10) || read_u64(fp, fbuf, m->nf * 9) ||
                  read_u64(fp, nbuf, m->nn * 4);
        if (bad) { free(cbuf); free(fbuf); free(nbuf); goto fail; }
        m->cell_faces = (uint64_t *)malloc(sizeof(uint64_t) * m->nc * 4);
        m->cell_nodes = (uint64_t *)malloc(sizeof(uint64_t) * m->nc * 4);
        m->cell_gid = (uint64_t *)malloc(sizeof(uint64_t) * m->nc);
        m->cell_mat = (uint64_t *)malloc(sizeof(uint64_t) * m->nc);
        for (uint64_t c = 0; c < m->nc; c++) {
            for (int k = 0; k < 4; k++) {
                m->cell_faces[c * 4 + k] = cbuf[c * 10 + k];
                m->cell_nodes[c * 4 + k] = cbuf[c * 10 + 4 + k];
            }
            m->cell_gid[c] = cbuf[c * 10 + 8];
            m->cell_mat[c] = cbuf[c * 10 + 9];
        }
        m->face_cells = (uint64_t *)malloc(sizeof(uint64_t) * m->nf * 2);
        m->face_nodes = (uint64_t *)malloc(sizeof(uint64_t) * m->nf * 3);
        m->face_btype = (uint64_t *)malloc(sizeof(uint64_t) * m->nf);
        m->face_gid = (uint64_t *)malloc(sizeof(uint64_t) * m->nf);
        m->face_part = (uint64_t *)malloc(sizeof(uint64_t) * m->nf * 2);
        for (uint64_t f = 0; f < m->nf; f++) {
            m->face_cells[f * 2 + 0] = fbuf[f * 9 + 0];
            m->face_cells[f * 2 + 1] = fbuf[f * 9 + 1];
            for (int k = 0; k < 3; k++) m->face_nodes[f * 3 + k] = fbuf[f * 9 + 2 + k];
            m->face_gid[f] = fbuf[f * 9 + 5];
            m->face_part[f * 2 + 0] = fbuf[f * 9 + 6];
            m->face_part[f * 2 + 1] = fbuf[f * 9 + 7];
            m->face_btype[f] = fbuf[f * 9 + 8];
        }
        m->coords = (double *)malloc(sizeof(double) * m->nn * 3);
        for (uint64_t n = 0; n < m->nn; n++)
            memcpy(&m->coords[n * 3], &nbuf[n * 4], 3 * sizeof(double));
        free(cbuf); free(fbuf); free(nbuf);
    }
    fclose(fp);
    fp = NULL;

    /* adjacency and local face numbering (src/TychoMeshIO.cc:196-227) */
    uint64_t nc = m->nc;
    m->adj_cell = (uint64_t *)malloc(sizeof(uint64_t) * nc * 4);
    m->adj_face = (uint64_t *)malloc(sizeof(uint64_t) * nc * 4);
    m->side = (uint64_t *)malloc(sizeof(uint64_t) * nc * 4);
    uint64_t *handle = (uint64_t *)malloc(sizeof(uint64_t) * nc * 4);
    m->nsides = 0;
    for (uint64_t c = 0; c < nc; c++) {
        for (uint64_t fi = 0; fi < 4; fi++) {
            uint64_t face = m->cell_faces[c * 4 + fi];
            if (face >= m->nf) { free(handle); goto fail; }
            uint64_t lf = lface_index(&m->cell_nodes[c * 4], &m->face_nodes[face * 3]);
            if (lf == OR_NONE) { free(handle); goto fail; }
            handle[c * 4 + lf] = fi;
            if (m->face_btype[face] != 2) {
                m->adj_cell[c * 4 + lf] = OR_NONE;
                m->adj_face[c * 4 + lf] = OR_NONE;
                m->nsides++;
            } else {
                uint64_t c1 = m->face_cells[face * 2], c2 = m->face_cells[face * 2 + 1];
                uint64_t adj = (c1 == c) ? c2 : c1;
                if (adj >= nc) { free(handle); goto fail; }
                m->adj_cell[c * 4 + lf] = adj;
                m->adj_face[c * 4 + lf] = lface_index(&m->cell_nodes[adj * 4], &m->face_nodes[face * 3]);
            }
        }
    }
    /* side numbering and global ids (src/TychoMeshIO.cc:228-248), the
       partition across each face (src/TychoMeshIO.cc:250-262) */
    m->side_gid = (uint64_t *)malloc(sizeof(uint64_t) * (m->nsides ? m->nsides : 1));
    m->adj_rank = (uint64_t *)malloc(sizeof(uint64_t) * nc * 4);
    {
        uint64_t s = 0;
        for (uint64_t c = 0; c < nc; c++)
            for (uint64_t f = 0; f < 4; f++) {
                uint64_t face = m->cell_faces[c * 4 + handle[c * 4 + f]];
                uint64_t p1 = m->face_part[face * 2], p2 = m->face_part[face * 2 + 1];
                m->adj_rank[c * 4 + f] = (p1 == m->part) ? p2 : p1;
                if (m->adj_cell[c * 4 + f] == OR_NONE) {
                    m->side_gid[s] = m->face_gid[face];
                    m->side[c * 4 + f] = s++;
                } else {
                    m->side[c * 4 + f] = OR_NONE;
                }
            }
    }
    /* faceToCellVrtx / cellToFaceVrtx (src/TychoMeshIO.cc:273-296): the face
       vertex index is the position of the node in the face record. */
    m->f2c = (uint64_t *)malloc(sizeof(uint64_t) * nc * 12);
    m->c2f = (uint64_t *)malloc(sizeof(uint64_t) * nc * 16);
    for (uint64_t i = 0; i < nc * 16; i++) m->c2f[i] = OR_NONE;
    for (uint64_t c = 0; c < nc; c++)
        for (uint64_t f = 0; f < 4; f++) {
            uint64_t face = m->cell_faces[c * 4 + handle[c * 4 + f]];
            for (uint64_t k = 0; k < 3; k++)
                for (uint64_t cv = 0; cv < 4; cv++)
                    if (m->face_nodes[face * 3 + k] == m->cell_nodes[c * 4 + cv]) {
                        m->f2c[(c * 4 + f) * 3 + k] = cv;
                        m->c2f[(c * 4 + f) * 4 + cv] = k;
                    }
        }
    free(handle);

    /* volumes, areas, outward normals (src/TychoMesh.cc:200-210, :214-220) */
    m->volume = (double *)malloc(sizeof(double) * nc);
    m->area = (double *)malloc(sizeof(double) * nc * 4);
    m->normal = (double *)malloc(sizeof(double) * nc * 12);
    for (uint64_t c = 0; c < nc; c++) {
        double cp[4][3], fp3[3][3];
        for (int v = 0; v < 4; v++)
            for (int d = 0; d < 3; d++) cp[v][d] = m->coords[m->cell_nodes[c * 4 + v] * 3 + d];
        m->volume[c] = tet_volume(cp);
        for (int f = 0; f < 4; f++) {
            for (int k = 0; k < 3; k++) {
                uint64_t cv = m->f2c[(c * 4 + f) * 3 + k];
                for (int d = 0; d < 3; d++) fp3[k][d] = cp[cv][d];
            }
            m->area[c * 4 + f] = tri_area(fp3);
            face_normal(fp3, cp, &m->normal[(c * 4 + f) * 3]);
        }
    }
    /* neighbor vertices (src/TychoMesh.cc:244-259) */
    m->nbr_vrtx = (uint64_t *)malloc(sizeof(uint64_t) * nc * 12);
    for (uint64_t c = 0; c < nc; c++)
        for (uint64_t f = 0; f < 4; f++)
            for (uint64_t k = 0; k < 3; k++) {
                uint64_t adj = m->adj_cell[c * 4 + f];
                if (adj == OR_NONE) { m->nbr_vrtx[(c * 4 + f) * 3 + k] = OR_NONE; continue; }
                uint64_t node = m->cell_nodes[c * 4 + m->f2c[(c * 4 + f) * 3 + k]];
                uint64_t nv = 0;
                for (uint64_t v = 0; v < 4; v++)
                    if (m->cell_nodes[adj * 4 + v] == node) { nv = v; break; }
                m->nbr_vrtx[(c * 4 + f) * 3 + k] = nv;
            }
    return m;
fail:
    if (fp) fclose(fp);
    om_free(m);
    return NULL;
}

uint64_t om_ncells(const OMesh *m) { return m->nc; }
uint64_t om_nnodes(const OMesh *m) { return m->nn; }
uint64_t om_nsides(const OMesh *m) { return m->nsides; }

/* Copies the integer and geometry tables out (any pointer may be NULL). */
void om_tables(const OMesh *m, uint64_t *adj_cell, uint64_t *nbr_vrtx, uint64_t *f2c,
               uint64_t *c2f, uint64_t *cell_nodes, double *volume, double *area,
               double *normal, uint64_t *side, uint64_t *cell_gid)
{
    uint64_t nc = m->nc;
    if (adj_cell) memcpy(adj_cell, m->adj_cell, nc * 4 * 8);
    if (nbr_vrtx) memcpy(nbr_vrtx, m->nbr_vrtx, nc * 12 * 8);
    if (f2c) memcpy(f2c, m->f2c, nc * 12 * 8);
    if (c2f) memcpy(c2f, m->c2f, nc * 16 * 8);
    if (cell_nodes) memcpy(cell_nodes, m->cell_nodes, nc * 4 * 8);
    if (volume) memcpy(volume, m->volume, nc * 8);
    if (area) memcpy(area, m->area, nc * 4 * 8);
    if (normal) memcpy(normal, m->normal, nc * 12 * 8);
    if (side) memcpy(side, m->side, nc * 4 * 8);
    if (cell_gid) memcpy(cell_gid, m->cell_gid, nc * 8);
}

void om_node_coords(const OMesh *m, double *out) { memcpy(out, m->coords, m->nn * 24); }

OMesh *om_load_pmesh(const char *path) { return om_load_pmesh_part(path, -1); }

/* partition, partition count; adjRank (c,4) and the sides' global ids (any
   pointer may be NULL). */
void om_partition(const OMesh *m, uint64_t *part, uint64_t *nparts, uint64_t *adj_rank, uint64_t *side_gid)
{
    if (part) *part = m->part;
    if (nparts) *nparts = m->nparts;
    if (adj_rank) memcpy(adj_rank, m->adj_rank, m->nc * 4 * 8);
    if (side_gid) memcpy(side_gid, m->side_gid, m->nsides * 8);
}

/* ------------------------------------------------------------------------ */
/* Quadrature (src/Quadrature.cc:150-244)                                    */
/* ------------------------------------------------------------------------ */

/* Fills xi, eta, mu, w (each 2*N*N) and returns the number of angles, or -1. */
int oq_quadrature(int sn, double *xi, double *eta, double *mu, double *w)
{
    const double *gn, *gw;
    if (tycho_gl_table(sn, &gn, &gw) != 0) return -1;
    for (int i = 0; i < sn; i++)
        for (int k = 0; k < 2 * sn; k++) {
            double phi = (2.0 * OR_PI) / (2 * sn) * (k + 0.5);
            int idx = i * 2 * sn + k;
            xi[idx] = sqrt(1.0 - gn[i] * gn[i]) * cos(phi);
            eta[idx] = sqrt(1.0 - gn[i] * gn[i]) * sin(phi);
            mu[idx] = gn[i];
            w[idx] = gw[i] * (2.0 * OR_PI) / (2 * sn);
        }
    return 2 * sn * sn;
}

/* ------------------------------------------------------------------------ */
/* Sweep context                                                            */
/* ------------------------------------------------------------------------ */

typedef struct {
    const OMesh *m;
    int A, G;
    double *xi, *eta, *mu, *w;
    double *odn;        /* (c,f,a): omega.n, src/TychoMesh.cc:212-223 */
    uint32_t *order;    /* per angle: cells in a topological order, (a, Nc) */
    uint32_t *tlevel;   /* (a, c): longest upwind chain */
    uint32_t *ndep;     /* (a, c): dependency count, src/GraphTraverser.cc:442-458 */
    int cyclic;         /* 1 if some angle's graph has a cycle */
    int gauss_elim;     /* 0 Original (pivoting), 1 NoPivot, 2 CramerGlu, 3 CramerIntel
                           (src/Global.hh:99-105) */
} OCtx;

void oc_free(OCtx *x)
{
    if (!x) return;
    free(x->xi); free(x->eta); free(x->mu); free(x->w); free(x->odn);
    free(x->order); free(x->tlevel); free(x->ndep);
    free(x);
}

static int is_incoming(const OCtx *x, uint64_t c, int f, int a)
{
    /* src/TychoMesh.hh:107-110 */
    return !(x->odn[((size_t)c * 4 + f) * x->A + a] > 0);
}

/* The visiting order is built on flux-carrying faces only: a face with
   omega.n == 0 exactly contributes nothing to the cell solve
   (src/Transport.cc:113, :184), but is_incoming() holds for it on both
   sides, a two-cycle on which the reference's traversal never finishes. */
static int is_upwind(const OCtx *x, uint64_t c, int f, int a)
{
    return x->odn[((size_t)c * 4 + f) * x->A + a] < 0;
}

static int is_downwind(const OCtx *x, uint64_t c, int f, int a)
{
    return x->odn[((size_t)c * 4 + f) * x->A + a] > 0;
}

/* Builds the context: quadrature, omega.n, per-angle topological orders and
   t-levels (Kahn's algorithm on the upwind graph of src/GraphTraverser.cc). */
OCtx *oc_create(const OMesh *m, int sn, int G)
{
    OCtx *x = (OCtx *)calloc(1, sizeof(OCtx));
    x->m = m; x->G = G; x->gauss_elim = 1;
    int A = 2 * sn * sn;
    x->A = A;
    x->xi = (double *)malloc(8 * A); x->eta = (double *)malloc(8 * A);
    x->mu = (double *)malloc(8 * A); x->w = (double *)malloc(8 * A);
    if (oq_quadrature(sn, x->xi, x->eta, x->mu, x->w) != A) { oc_free(x); return NULL; }
    uint64_t nc = m->nc;
    x->odn = (double *)malloc(sizeof(double) * nc * 4 * A);
    for (uint64_t c = 0; c < nc; c++)
        for (int f = 0; f < 4; f++) {
            const double *n = &m->normal[(c * 4 + f) * 3];
            for (int a = 0; a < A; a++)
                x->odn[(c * 4 + f) * A + a] = x->xi[a] * n[0] + x->eta[a] * n[1] + x->mu[a] * n[2];
        }
    x->order = (uint32_t *)malloc(sizeof(uint32_t) * nc * A);
    x->tlevel = (uint32_t *)malloc(sizeof(uint32_t) * nc * A);
    x->ndep = (uint32_t *)malloc(sizeof(uint32_t) * nc * A);
    int cyc = 0;
    #pragma omp parallel for schedule(dynamic) reduction(|:cyc)
    for (int a = 0; a < A; a++) {
        uint32_t *dep = &x->ndep[(size_t)a * nc];
        uint32_t *lev = &x->tlevel[(size_t)a * nc];
        uint32_t *ord = &x->order[(size_t)a * nc];
        uint32_t *cnt = (uint32_t *)malloc(sizeof(uint32_t) * nc);
        size_t head = 0, tail = 0;
        for (uint64_t c = 0; c < nc; c++) {
            uint32_t d = 0, u = 0;
            for (int f = 0; f < 4; f++) {
                if (m->adj_cell[c * 4 + f] == OR_NONE) continue;
                if (is_incoming(x, c, f, a)) d++;
                if (is_upwind(x, c, f, a)) u++;
            }
            dep[c] = d; cnt[c] = u; lev[c] = 0;
            if (u == 0) ord[tail++] = (uint32_t)c;
        }
        while (head < tail) {
            uint64_t c = ord[head++];
            for (int f = 0; f < 4; f++) {
                uint64_t adj = m->adj_cell[c * 4 + f];
                if (adj == OR_NONE || !is_downwind(x, c, f, a)) continue;
                if (lev[adj] < lev[c] + 1) lev[adj] = lev[c] + 1;
                if (--cnt[adj] == 0) ord[tail++] = (uint32_t)adj;
            }
        }
        if (tail != nc) cyc |= 1;
        free(cnt);
    }
    x->cyclic = cyc;
    return x;
}

int oc_num_angles(const OCtx *x) { return x->A; }
int oc_cyclic(const OCtx *x) { return x->cyclic; }
void oc_set_gauss_elim(OCtx *x, int kind) { x->gauss_elim = kind; }

void oc_quadrature(const OCtx *x, double *xi, double *eta, double *mu, double *w)
{
    memcpy(xi, x->xi, 8 * x->A); memcpy(eta, x->eta, 8 * x->A);
    memcpy(mu, x->mu, 8 * x->A); memcpy(w, x->w, 8 * x->A);
}

/* omega.n in the reference's Mat3(angle, cell, face) order: ((f*Nc)+c)*A + a. */
void oc_omega_dot_n(const OCtx *x, double *out)
{
    uint64_t nc = x->m->nc;
    for (uint64_t c = 0; c < nc; c++)
        for (int f = 0; f < 4; f++)
            for (int a = 0; a < x->A; a++)
                out[((size_t)f * nc + c) * x->A + a] = x->odn[(c * 4 + f) * x->A + a];
}

/* t-levels and dependency counts, (a, c) order. */
void oc_levels(const OCtx *x, uint32_t *tlevel, uint32_t *ndep)
{
    size_t n = (size_t)x->A * x->m->nc;
    if (tlevel) memcpy(tlevel, x->tlevel, 4 * n);
    if (ndep) memcpy(ndep, x->ndep, 4 * n);
}

/* b-levels: the longest downwind chain, what Priorities' BLevelData computes
   on the backward traversal (src/Priorities.cc:59-164, :396-405).  Visits
   cells in reverse topological order. (a, c) order. */
void oc_blevels(const OCtx *x, uint32_t *blev)
{
    uint64_t nc = x->m->nc;
    for (int a = 0; a < x->A; a++) {
        const uint32_t *ord = &x->order[(size_t)a * nc];
        uint32_t *b = &blev[(size_t)a * nc];
        for (uint64_t i = nc; i-- > 0;) {
            uint64_t c = ord[i];
            uint32_t best = 0;
            for (int f = 0; f < 4; f++) {
                uint64_t adj = x->m->adj_cell[c * 4 + f];
                if (adj == OR_NONE || is_incoming(x, c, f, a)) continue;
                if (b[adj] + 1 > best) best = b[adj] + 1;
            }
            b[c] = best;
        }
    }
}

/* Gaussian elimination variants (src/Transport.cc:277-410). */
static void gauss_original(double A[4][4], double b[4])
{
    const int n = 4;
    for (int column = 0; column < n - 1; ++column) {
        int rowmax = column;
        double colmax = fabs(A[column][column]);
        for (int row = column + 1; row < n; ++row) {
            double t = fabs(A[row][column]);
            if (t > colmax) { rowmax = row; colmax = t; }
        }
        if (rowmax != column) {
            for (int c2 = 0; c2 < n; ++c2) {
                double t = A[rowmax][c2]; A[rowmax][c2] = A[column][c2]; A[column][c2] = t;
            }
            double t = b[rowmax]; b[rowmax] = b[column]; b[column] = t;
        }
        A[column][column] = 1. / A[column][column];
        for (int row = column + 1; row < n; ++row) A[row][column] *= A[column][column];
        for (int c2 = 0; c2 <= column; ++c2)
            for (int row = c2 + 1; row < n; ++row)
                A[row][column + 1] -= A[row][c2] * A[c2][column + 1];
    }
    A[n - 1][n - 1] = 1. / A[n - 1][n - 1];
    for (int column = 0; column < n - 1; ++column)
        for (int row = column + 1; row < n; ++row) b[row] -= A[row][column] * b[column];
    for (int column = n - 1; column >= 0; --column) {
        b[column] *= A[column][column];
        for (int row = column - 1; row >= 0; --row) b[row] -= A[row][column] * b[column];
    }
}

static void gauss_nopivot(double A[4][4], double b[4])
{
    double t;
    t = 1.0 / A[0][0];
    A[0][0] = 1.0; A[0][1] = A[0][1] * t; A[0][2] = A[0][2] * t; A[0][3] = A[0][3] * t;
    b[0] = b[0] * t;
    for (int r = 1; r < 4; r++) {
        t = A[r][0];
        A[r][0] = 0.0;
        A[r][1] = A[r][1] - A[0][1] * t;
        A[r][2] = A[r][2] - A[0][2] * t;
        A[r][3] = A[r][3] - A[0][3] * t;
        b[r] = b[r] - b[0] * t;
    }
    t = 1.0 / A[1][1];
    A[1][1] = 1.0; A[1][2] = A[1][2] * t; A[1][3] = A[1][3] * t; b[1] = b[1] * t;
    for (int r = 2; r < 4; r++) {
        t = A[r][1];
        A[r][1] = 0.0;
        A[r][2] = A[r][2] - A[1][2] * t;
        A[r][3] = A[r][3] - A[1][3] * t;
        b[r] = b[r] - b[1] * t;
    }
    t = 1.0 / A[2][2];
    A[2][2] = 1.0; A[2][3] = A[2][3] * t; b[2] = b[2] * t;
    t = A[3][2];
    A[3][2] = 0.0; A[3][3] = A[3][3] - A[2][3] * t; b[3] = b[3] - b[2] * t;
    b[3] = b[3] / A[3][3];
    b[2] = b[2] - A[2][3] * b[3];
    b[1] = b[1] - A[1][3] * b[3] - A[1][2] * b[2];
    b[0] = b[0] - A[0][3] * b[3] - A[0][2] * b[2] - A[0][1] * b[1];
}

/* gaussElim4 CramerGlu (src/Transport.cc:414-557): the inverse by cofactors,
   then x = inv b.  inv[4a + b] is the (b, a) cofactor, (-1)^(a+b) times the
   minor without row b and column a, expanded along its first column c0 over
   the rows r in increasing order, each row's 2x2 minor written as
   m[r][c0] m[r'][c1] m[r''][c2] - m[r][c0] m[r'][c2] m[r''][c1] (r' < r'',
   c0 < c1 < c2), every product left to right and the six terms summed left
   to right: the operation order the reference's expressions have. */
static void gauss_cramer_glu(double A[4][4], double b[4])
{
    double inv[16], det;
    for (int a = 0; a < 4; a++)
        for (int bb = 0; bb < 4; bb++) {
            int rows[3], cols[3], nr = 0, ncl = 0;
            for (int r = 0; r < 4; r++) if (r != bb) rows[nr++] = r;
            for (int c = 0; c < 4; c++) if (c != a) cols[ncl++] = c;
            double sign = ((a + bb) & 1) ? -1.0 : 1.0, acc = 0.0;
            for (int k = 0; k < 3; k++) {
                int r = rows[k], r1 = rows[k == 0 ? 1 : 0], r2 = rows[k == 2 ? 1 : 2];
                double sg = (k & 1) ? -sign : sign;
                double t1 = A[r][cols[0]] * A[r1][cols[1]] * A[r2][cols[2]];
                double t2 = A[r][cols[0]] * A[r1][cols[2]] * A[r2][cols[1]];
                if (k == 0) acc = sg > 0 ? t1 : -t1;
                else acc = sg > 0 ? acc + t1 : acc - t1;
                acc = sg > 0 ? acc - t2 : acc + t2;
            }
            inv[4 * a + bb] = acc;
        }
    det = A[0][0] * inv[0] + A[0][1] * inv[4] + A[0][2] * inv[8] + A[0][3] * inv[12];
    det = 1.0 / det;
    for (int i = 0; i < 16; i++) inv[i] = inv[i] * det;
    double x[4];
    for (int r = 0; r < 4; r++) x[r] = inv[4 * r] * b[0] + inv[4 * r + 1] * b[1] + inv[4 * r + 2] * b[2] + inv[4 * r + 3] * b[3];
    for (int r = 0; r < 4; r++) b[r] = x[r];
}

/* gaussElim4 CramerIntel (src/Transport.cc:559-677): the scalar form of
   Intel's SSE 4x4 inverse (application note "Streaming SIMD Extensions -
   Inverse of 4x4 Matrix").  src is A column-major; pairs of products of two
   rows of src (tmp), cofactors as (three tmp x src products) minus (three
   more), determinant, scaling, x = inv b.  The tables give each cofactor's
   (tmp, src) pairs in the order the reference sums them. */
static const unsigned char kIntelCof[16][6][2] = {
    {{0, 5}, {3, 6}, {4, 7}, {1, 5}, {2, 6}, {5, 7}},       {{1, 4}, {6, 6}, {9, 7}, {0, 4}, {7, 6}, {8, 7}},
    {{2, 4}, {7, 5}, {10, 7}, {3, 4}, {6, 5}, {11, 7}},     {{5, 4}, {8, 5}, {11, 6}, {4, 4}, {9, 5}, {10, 6}},
    {{1, 1}, {2, 2}, {5, 3}, {0, 1}, {3, 2}, {4, 3}},       {{0, 0}, {7, 2}, {8, 3}, {1, 0}, {6, 2}, {9, 3}},
    {{3, 0}, {6, 1}, {11, 3}, {2, 0}, {7, 1}, {10, 3}},     {{4, 0}, {9, 1}, {10, 2}, {5, 0}, {8, 1}, {11, 2}},
    {{0, 13}, {3, 14}, {4, 15}, {1, 13}, {2, 14}, {5, 15}}, {{1, 12}, {6, 14}, {9, 15}, {0, 12}, {7, 14}, {8, 15}},
    {{2, 12}, {7, 13}, {10, 15}, {3, 12}, {6, 13}, {11, 15}}, {{5, 12}, {8, 13}, {11, 14}, {4, 12}, {9, 13}, {10, 14}},
    {{2, 10}, {5, 11}, {1, 9}, {4, 11}, {0, 9}, {3, 10}},   {{8, 11}, {0, 8}, {7, 10}, {6, 10}, {9, 11}, {1, 8}},
    {{6, 9}, {11, 11}, {3, 8}, {10, 11}, {2, 8}, {7, 9}},   {{10, 10}, {4, 8}, {9, 9}, {8, 9}, {11, 10}, {5, 8}}};
/* column pairs (p, q) of the tmp products, in order: tmp[2k] = s[p] s[q'] ... */
static const unsigned char kIntelPairs[6][2] = {{2, 3}, {1, 3}, {1, 2}, {0, 3}, {0, 2}, {0, 1}};

static void gauss_cramer_intel(double A[4][4], double b[4])
{
    double src[16], dst[16], tmp[12], det;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) src[i + 4 * j] = A[i][j];
    for (int half = 0; half < 2; half++) {
        /* first half: rows 2, 3 of src (8..15); second: rows 0, 1 (0..7) */
        const int lo = half ? 0 : 8, hi = half ? 4 : 12;
        for (int k = 0; k < 6; k++) {
            const int p = kIntelPairs[k][0], q = kIntelPairs[k][1];
            tmp[2 * k] = src[lo + p] * src[hi + q];
            tmp[2 * k + 1] = src[lo + q] * src[hi + p];
        }
        for (int j = 8 * half; j < 8 * half + 8; j++) {
            const unsigned char(*t)[2] = kIntelCof[j];
            double plus = tmp[t[0][0]] * src[t[0][1]] + tmp[t[1][0]] * src[t[1][1]] + tmp[t[2][0]] * src[t[2][1]];
            double minus = tmp[t[3][0]] * src[t[3][1]] + tmp[t[4][0]] * src[t[4][1]] + tmp[t[5][0]] * src[t[5][1]];
            dst[j] = plus - minus;
        }
    }
    det = src[0] * dst[0] + src[1] * dst[1] + src[2] * dst[2] + src[3] * dst[3];
    det = 1 / det;
    for (int j = 0; j < 16; j++) dst[j] *= det;
    double x[4];
    for (int r = 0; r < 4; r++) x[r] = dst[4 * r] * b[0] + dst[4 * r + 1] * b[1] + dst[4 * r + 2] * b[2] + dst[4 * r + 3] * b[3];
    for (int r = 0; r < 4; r++) b[r] = x[r];
}

/* One (cell, angle) update: SweepData::update + Transport::populateLocalPsiBound
   + Transport::solve (src/SweepData.hh:139-174, src/Transport.cc:57-271,
   :687-776).  Source per (v,g): angular part (psi layout, may be NULL) plus
   isotropic part (phi layout, may be NULL); exactly one addition when both. */
static void cell_update(const OCtx *x, uint64_t c, int a, const double *src_ang,
                        const double *src_iso, const double *sigma_t, const double *psi_bound,
                        double *psi)
{
    const OMesh *m = x->m;
    const int A = x->A, G = x->G;
    double volume = m->volume[c];
    double area[4];
    for (int f = 0; f < 4; f++)
        area[f] = m->area[c * 4 + f] * x->odn[(c * 4 + f) * A + a];
    double sigma = sigma_t[c];
    for (int g = 0; g < G; g++) {
        double q[4];
        for (int v = 0; v < 4; v++) {
            if (src_ang && src_iso)
                q[v] = src_ang[(((size_t)c * A + a) * 4 + v) * G + g] + src_iso[((size_t)c * 4 + v) * G + g];
            else if (src_ang)
                q[v] = src_ang[(((size_t)c * A + a) * 4 + v) * G + g];
            else if (src_iso)
                q[v] = src_iso[((size_t)c * 4 + v) * G + g];
            else
                q[v] = 0.0;
        }
        /* calcSource (src/Transport.cc:57-72) */
        double b[4];
        b[0] = volume / 20.0 * (2.0 * q[0] + q[1] + q[2] + q[3]);
        b[1] = volume / 20.0 * (q[0] + 2.0 * q[1] + q[2] + q[3]);
        b[2] = volume / 20.0 * (q[0] + q[1] + 2.0 * q[2] + q[3]);
        b[3] = volume / 20.0 * (q[0] + q[1] + q[2] + 2.0 * q[3]);
        /* calcVolumeIntegrals (src/Transport.cc:78-103) */
        double M[4][4];
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++)
                M[i][j] = (i == j) ? area[i] / 12.0 + 2.0 * sigma * volume / 20.0
                                   : area[i] / 12.0 + 1.0 * sigma * volume / 20.0;
        /* calcOutgoingFlux (src/Transport.cc:109-168) */
        for (int f = 0; f < 4; f++) {
            if (!(area[f] > 0)) continue;
            for (int i = 0; i < 4; i++) {
                if (i == f) continue;
                for (int j = 0; j < 4; j++) {
                    if (j == f) continue;
                    M[i][j] += (i == j ? 2.0 : 1.0) * area[f] / 12.0;
                }
            }
        }
        /* populateLocalPsiBound + calcIncomingFlux (src/Transport.cc:740-776,
           :174-271).  Upwind psi at the neighbor vertex that shares cell
           vertex j; on a face whose neighbour is another partition, the
           boundary value psiBound(g, fv, a, side) (psi_bound non-NULL:
           PsiBoundData layout, src/PsiData.hh:253-262); vacuum (0) on mesh
           boundaries. */
        for (int f = 0; f < 4; f++) {
            if (!(area[f] < 0)) continue;
            double pn[4] = {0.0, 0.0, 0.0, 0.0};
            uint64_t adj = m->adj_cell[c * 4 + f];
            if (is_incoming(x, c, f, a) && adj != OR_NONE) {
                for (int j = 0; j < 4; j++) {
                    if (j == f) continue;
                    uint64_t fv = m->c2f[(c * 4 + f) * 4 + j];
                    uint64_t nv = m->nbr_vrtx[(c * 4 + f) * 3 + fv];
                    pn[j] = psi[(((size_t)adj * A + a) * 4 + nv) * G + g];
                }
            } else if (is_incoming(x, c, f, a) && psi_bound && m->adj_rank[c * 4 + f] != OR_NONE) {
                uint64_t side = m->side[c * 4 + f];
                for (int j = 0; j < 4; j++) {
                    if (j == f) continue;
                    uint64_t fv = m->c2f[(c * 4 + f) * 4 + j];
                    pn[j] = psi_bound[(((size_t)side * A + a) * 3 + fv) * G + g];
                }
            }
            for (int i = 0; i < 4; i++) {
                if (i == f) continue;
                for (int j = 0; j < 4; j++) {
                    if (j == f) continue;
                    b[i] -= (i == j ? 2.0 : 1.0) * area[f] / 12.0 * pn[j];
                }
            }
        }
        switch (x->gauss_elim) {
        case 0: gauss_original(M, b); break;
        case 2: gauss_cramer_glu(M, b); break;
        case 3: gauss_cramer_intel(M, b); break;
        default: gauss_nopivot(M, b); break;
        }
        for (int v = 0; v < 4; v++) psi[(((size_t)c * A + a) * 4 + v) * G + g] = b[v];
    }
}

/* psi = L^{-1} source: the full sweep (src/SweeperTraverse.cc:82-89). */
int oc_sweep(const OCtx *x, const double *src_ang, const double *src_iso,
             const double *sigma_t, double *psi)
{
    if (x->cyclic) return -1;
    uint64_t nc = x->m->nc;
    #pragma omp parallel for schedule(dynamic)
    for (int a = 0; a < x->A; a++) {
        const uint32_t *ord = &x->order[(size_t)a * nc];
        for (uint64_t i = 0; i < nc; i++) cell_update(x, ord[i], a, src_ang, src_iso, sigma_t, NULL, psi);
    }
    return 0;
}

/* One partition's local sweep with its incoming partition-boundary values:
   Util::sweepLocal(psi, source, psiBound) under a GraphTraverser built
   without communication (src/Util.cc:138-145, src/GraphTraverser.cc:442-458:
   only faces to cells of this partition order the sweep). */
int oc_sweep_local(const OCtx *x, const double *src_ang, const double *src_iso,
                   const double *sigma_t, const double *psi_bound, double *psi)
{
    if (x->cyclic) return -1;
    uint64_t nc = x->m->nc;
    #pragma omp parallel for schedule(dynamic)
    for (int a = 0; a < x->A; a++) {
        const uint32_t *ord = &x->order[(size_t)a * nc];
        for (uint64_t i = 0; i < nc; i++) cell_update(x, ord[i], a, src_ang, src_iso, sigma_t, psi_bound, psi);
    }
    return 0;
}

/* phi = sum_a w_a psi_a in angle order (src/Util.cc:85-97). */
void oc_psi_to_phi(const OCtx *x, const double *psi, double *phi)
{
    uint64_t nc = x->m->nc;
    int A = x->A, G = x->G;
    #pragma omp parallel for
    for (int64_t c = 0; c < (int64_t)nc; c++) {
        for (int i = 0; i < 4 * G; i++) phi[(size_t)c * 4 * G + i] = 0.0;
        for (int a = 0; a < A; a++)
            for (int v = 0; v < 4; v++)
                for (int g = 0; g < G; g++)
                    phi[((size_t)c * 4 + v) * G + g] += psi[(((size_t)c * A + a) * 4 + v) * G + g] * x->w[a];
    }
}

/* Scattering source S phi (src/Util.cc:118-130, :151-159).  With
   scat == NULL scattering is within-group: sigma_s[c]/(4 pi) * phi, as the
   reference computes it.  Otherwise group-to-group:
   iso(c,v,g) = sum over g' with scat[g*G+g'] != 0, in increasing g', of
   (sigma_s[c] * scat[g*G+g'] / (4 pi)) * phi(c,v,g'), starting from 0. */
void oc_scatter(const OCtx *x, const double *sigma_s, const double *scat,
                const double *phi, double *iso)
{
    uint64_t nc = x->m->nc;
    int G = x->G;
    #pragma omp parallel for
    for (int64_t c = 0; c < (int64_t)nc; c++)
        for (int v = 0; v < 4; v++)
            for (int g = 0; g < G; g++) {
                size_t i = ((size_t)c * 4 + v) * G + g;
                if (!scat) {
                    iso[i] = sigma_s[c] / (4.0 * OR_PI) * phi[i];
                } else {
                    double s = 0.0;
                    for (int gp = 0; gp < G; gp++) {
                        double k = scat[g * G + gp];
                        if (k == 0.0) continue;
                        s += sigma_s[c] * k / (4.0 * OR_PI) * phi[((size_t)c * 4 + v) * G + gp];
                    }
                    iso[i] = s;
                }
            }
}

/* Source iteration (src/SourceIteration.cc:127-207): phi starts at 0 (psi is
   zeroed by SweeperTraverse::solve), each step sweeps Q + S phi_old, stops
   when the L1 relative change of phi is <= err_max or after iter_max steps.
   The fixed source is angular (q_ang) or isotropic (q_iso); psi, phi out.
   Returns the number of iterations. */
int oc_source_iteration(const OCtx *x, const double *sigma_t, const double *sigma_s,
                        const double *scat, const double *q_ang, const double *q_iso,
                        int iter_max, double err_max, double *psi, double *phi,
                        double *err_out)
{
    uint64_t nc = x->m->nc;
    size_t nphi = (size_t)nc * 4 * x->G;
    double *phi_old = (double *)malloc(8 * nphi);
    double *iso = (double *)malloc(8 * nphi);
    memset(psi, 0, 8 * nphi * x->A);
    oc_psi_to_phi(x, psi, phi);
    int iter = 0;
    double error = 1.0;
    while (iter < iter_max && error > err_max) {
        memcpy(phi_old, phi, 8 * nphi);
        oc_scatter(x, sigma_s, scat, phi_old, iso);
        if (q_iso)
            for (size_t i = 0; i < nphi; i++) iso[i] = q_iso[i] + iso[i];
        if (oc_sweep(x, q_ang, iso, sigma_t, psi) != 0) { iter = -1; break; }
        oc_psi_to_phi(x, psi, phi);
        double norm = 0.0;
        error = 0.0;
        for (size_t i = 0; i < nphi; i++) {
            error += fabs(phi[i] - phi_old[i]);
            norm += fabs(phi[i]);
        }
        error = error / norm;
        ++iter;
    }
    if (err_out) *err_out = error;
    free(phi_old); free(iso);
    return iter;
}

/* ------------------------------------------------------------------------ */
/* Krylov path (src/SourceIteration.cc:76-114, :216-285) with a restarted    */
/* GMRES(m) in place of PETSc's KSPGMRES (absent here): modified            */
/* Gram-Schmidt, Givens rotations, zero initial guess, stop when the        */
/* residual norm <= rtol * ||b||.                                           */
/* ------------------------------------------------------------------------ */

typedef struct {
    const OCtx *x;
    const double *sigma_t, *sigma_s, *scat;
    double *psi, *iso;
} LhsData;

/* b = (I - D L^{-1} M S) x */
static int lhs_apply(LhsData *d, const double *xv, double *bv)
{
    const OCtx *x = d->x;
    size_t nphi = (size_t)x->m->nc * 4 * x->G;
    oc_scatter(x, d->sigma_s, d->scat, xv, d->iso);
    if (oc_sweep(x, NULL, d->iso, d->sigma_t, d->psi) != 0) return -1;
    oc_psi_to_phi(x, d->psi, bv);
    for (size_t i = 0; i < nphi; i++) bv[i] = xv[i] - bv[i];
    return 0;
}

static double dot(const double *a, const double *b, size_t n)
{
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

int oc_krylov(const OCtx *x, const double *sigma_t, const double *sigma_s,
              const double *scat, const double *q_ang, const double *q_iso,
              int restart, int iter_max, double rtol, double *psi, double *phi,
              double *rnorm_out)
{
    size_t n = (size_t)x->m->nc * 4 * x->G;
    int m = restart;
    LhsData d = {x, sigma_t, sigma_s, scat, psi, (double *)malloc(8 * n)};
    double *b = (double *)malloc(8 * n);
    double *V = (double *)malloc(8 * n * (m + 1));
    double *H = (double *)calloc((size_t)(m + 1) * m, 8);
    double *cs = (double *)malloc(8 * m), *sn = (double *)malloc(8 * m);
    double *gv = (double *)malloc(8 * (m + 1)), *y = (double *)malloc(8 * m);
    double *r = (double *)malloc(8 * n);
    int its = 0, status = 0;
    double rnorm = 0.0;

    /* b = D L^{-1} Q */
    if (oc_sweep(x, q_ang, q_iso, sigma_t, psi) != 0) { status = -1; goto done; }
    oc_psi_to_phi(x, psi, b);
    double bnorm = sqrt(dot(b, b, n));
    for (size_t i = 0; i < n; i++) phi[i] = 0.0;
    if (bnorm == 0.0) goto final;
    for (;;) {
        /* r = b - A phi */
        if (its == 0) memcpy(r, b, 8 * n);
        else {
            if (lhs_apply(&d, phi, r) != 0) { status = -1; goto done; }
            for (size_t i = 0; i < n; i++) r[i] = b[i] - r[i];
        }
        double beta = sqrt(dot(r, r, n));
        rnorm = beta;
        if (beta <= rtol * bnorm || its >= iter_max) break;
        for (size_t i = 0; i < n; i++) V[i] = r[i] / beta;
        memset(gv, 0, 8 * (m + 1));
        gv[0] = beta;
        int k;
        for (k = 0; k < m && its < iter_max; k++) {
            double *vk1 = &V[n * (k + 1)];
            if (lhs_apply(&d, &V[n * k], vk1) != 0) { status = -1; goto done; }
            its++;
            for (int j = 0; j <= k; j++) {
                double h = dot(vk1, &V[n * j], n);
                H[j * m + k] = h;
                for (size_t i = 0; i < n; i++) vk1[i] -= h * V[n * j + i];
            }
            double hn = sqrt(dot(vk1, vk1, n));
            H[(k + 1) * m + k] = hn;
            if (hn != 0.0) for (size_t i = 0; i < n; i++) vk1[i] /= hn;
            for (int j = 0; j < k; j++) {
                double t = cs[j] * H[j * m + k] + sn[j] * H[(j + 1) * m + k];
                H[(j + 1) * m + k] = -sn[j] * H[j * m + k] + cs[j] * H[(j + 1) * m + k];
                H[j * m + k] = t;
            }
            double den = sqrt(H[k * m + k] * H[k * m + k] + hn * hn);
            cs[k] = H[k * m + k] / den; sn[k] = hn / den;
            H[k * m + k] = den; H[(k + 1) * m + k] = 0.0;
            gv[k + 1] = -sn[k] * gv[k];
            gv[k] = cs[k] * gv[k];
            rnorm = fabs(gv[k + 1]);
            if (rnorm <= rtol * bnorm) { k++; break; }
        }
        for (int i = k - 1; i >= 0; i--) {
            double s = gv[i];
            for (int j = i + 1; j < k; j++) s -= H[i * m + j] * y[j];
            y[i] = s / H[i * m + i];
        }
        for (int j = 0; j < k; j++)
            for (size_t i = 0; i < n; i++) phi[i] += y[j] * V[n * j + i];
        if (rnorm <= rtol * bnorm || its >= iter_max) {
            /* true residual for the report */
            if (lhs_apply(&d, phi, r) != 0) { status = -1; goto done; }
            for (size_t i = 0; i < n; i++) r[i] = b[i] - r[i];
            rnorm = sqrt(dot(r, r, n));
            break;
        }
    }
final:
    /* psi = L^{-1}(M S phi + Q) */
    oc_scatter(x, sigma_s, scat, phi, d.iso);
    if (q_iso) for (size_t i = 0; i < n; i++) d.iso[i] = q_iso[i] + d.iso[i];
    if (oc_sweep(x, q_ang, d.iso, sigma_t, psi) != 0) status = -1;
done:
    if (rnorm_out) *rnorm_out = rnorm;
    free(d.iso); free(b); free(V); free(H); free(cs); free(sn); free(gv); free(y); free(r);
    return status == 0 ? its : -1;
}

/* ------------------------------------------------------------------------ */
/* Problems                                                                  */
/* ------------------------------------------------------------------------ */

/* The reference's "hat" manufactured source on the [0,100]^3 cube
   (src/Problem.cc:47-82); sigma_t, sigma_s per cell. */
void oc_hat_source(const OCtx *x, const double *sigma_t, const double *sigma_s, double *src)
{
    const OMesh *m = x->m;
    const double cube = 100.0;
    int A = x->A, G = x->G;
    for (uint64_t c = 0; c < m->nc; c++)
        for (int a = 0; a < A; a++)
            for (int v = 0; v < 4; v++) {
                uint64_t node = m->cell_nodes[c * 4 + v];
                double px = m->coords[node * 3 + 0] - cube / 2.0;
                double py = m->coords[node * 3 + 1] - cube / 2.0;
                double pz = m->coords[node * 3 + 2] - cube / 2.0;
                double xi = x->xi[a], eta = x->eta[a], mu = x->mu[a];
                double r = sqrt(px * px + py * py + pz * pz);
                for (int g = 0; g < G; g++) {
                    double val = 0.0;
                    if (r <= 30.0)
                        val = -px / (30.0 * r) * xi - py / (30.0 * r) * eta - pz / (30.0 * r) * mu +
                              (sigma_t[c] - sigma_s[c]) * (1.0 - r / 30.0);
                    src[(((size_t)c * A + a) * 4 + v) * G + g] = val;
                }
            }
}

/* .psi writer (src/PsiData.cc:62-106): 32-byte name, u64 version, cells,
   angles, groups, then psi in global cell order. */
int oc_write_psi(const OCtx *x, const double *psi, const char *path)
{
    FILE *fp = fopen(path, "wb");
    if (!fp) return -1;
    char name[32] = "Tycho 2 Psi Output";
    uint64_t hdr[4] = {1, x->m->nc, (uint64_t)x->A, (uint64_t)x->G};
    fwrite(name, 1, 32, fp);
    fwrite(hdr, 8, 4, fp);
    size_t per = (size_t)x->A * 4 * x->G;
    for (uint64_t c = 0; c < x->m->nc; c++) {
        long off = (long)(64 + x->m->cell_gid[c] * per * 8);
        fseek(fp, off, SEEK_SET);
        fwrite(&psi[c * per], 8, per, fp);
    }
    fclose(fp);
    return 0;
}
