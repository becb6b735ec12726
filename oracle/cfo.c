/* CPU restatement of the reference's 3D SIMPLE hot path -- TEST ORACLE ONLY.
 *
 * Plain C11, FP64, serial; compile with -ffp-contract=off (oracle/Makefile).
 * Each routine cites the reference function it restates (paths relative to
 * the ChuanFlow source tree) and keeps its operation order, so its outputs
 * are bit-identical to the reference's own build wherever the reference is
 * itself deterministic.  The product (chuanflow_b200/) never uses this file.
 */
#define _POSIX_C_SOURCE 200809L
#include "cfo.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* errors                                                                    */
/* ------------------------------------------------------------------------ */

static char g_err[512];

static int fail(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return -1;
}

const char* cfo_last_error(void) { return g_err; }

/* ------------------------------------------------------------------------ */
/* Vector3 (src/common/include/cf/common/Vector.h:13-61)                     */
/* ------------------------------------------------------------------------ */

typedef struct { double x, y, z; } v3;

static inline v3 V3(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vneg(v3 a) { return V3(-a.x, -a.y, -a.z); }
static inline v3 vmul(v3 a, double s) { return V3(a.x * s, a.y * s, a.z * s); }
static inline v3 vdiv(v3 a, double s) { return V3(a.x / s, a.y / s, a.z / s); }
static inline double vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b)
{
    return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline double vmag(v3 a) { return sqrt(vdot(a, a)); }
static inline double vcomp(v3 a, int c) { return c == 0 ? a.x : (c == 1 ? a.y : a.z); }
static inline void vset(v3* a, int c, double v)
{
    if (c == 0) a->x = v;
    else if (c == 1) a->y = v;
    else a->z = v;
}
static inline v3 ld(const double* p, int64_t i) { return V3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
static inline void st(double* p, int64_t i, v3 v)
{
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}

/* std::max / std::min / std::clamp as libstdc++ defines them */
static inline double smax(double a, double b) { return (a < b) ? b : a; }
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double sclamp(double v, double lo, double hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }

static void* xcalloc(size_t n, size_t s)
{
    void* p = calloc(n ? n : 1, s);
    if (!p) { fprintf(stderr, "cfo: out of memory\n"); abort(); }
    return p;
}

/* ------------------------------------------------------------------------ */
/* blockMesh (src/3d/src/mesh/blockMesh.cpp:36-189)                         */
/* ------------------------------------------------------------------------ */

int cfo_block_counts(int64_t nx, int64_t ny, int64_t nz, int64_t out[4])
{
    if (nx <= 0 || ny <= 0 || nz <= 0) return fail("blockMesh: cell counts must be positive");
    out[0] = (nx + 1) * (ny + 1) * (nz + 1);
    out[1] = nx * ny * nz;
    out[3] = (nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1);
    out[2] = out[3] + 2 * (ny * nz + nx * nz + nx * ny);
    return 0;
}

typedef struct { int64_t key[4]; int64_t verts[4]; int64_t owner, nbr; } face_ref;

static void sort4(const int64_t* v, int64_t* k)
{
    for (int i = 0; i < 4; ++i) k[i] = v[i];
    for (int i = 1; i < 4; ++i)
        for (int j = i; j > 0 && k[j - 1] > k[j]; --j) { int64_t t = k[j]; k[j] = k[j - 1]; k[j - 1] = t; }
}

static uint64_t hash4(const int64_t* k)
{
    uint64_t h = 1469598103934665603ULL;
    for (int i = 0; i < 4; ++i) { h ^= (uint64_t)k[i]; h *= 1099511628211ULL; h ^= h >> 29; }
    return h;
}

int cfo_block_mesh(const double mn[3], const double mx[3], int64_t nx, int64_t ny, int64_t nz,
                   double* pts, int64_t* fOff, int64_t* fV, int64_t* own, int64_t* nbr,
                   int64_t* pStart, int64_t* pSize)
{
    int64_t cnt[4];
    if (cfo_block_counts(nx, ny, nz, cnt)) return -1;
#define PAT(i, j, k) ((i) + (nx + 1) * ((j) + (ny + 1) * (k)))
    for (int64_t k = 0; k <= nz; ++k)
        for (int64_t j = 0; j <= ny; ++j)
            for (int64_t i = 0; i <= nx; ++i)
            {
                const int64_t p = PAT(i, j, k);
                pts[3 * p] = mn[0] + (mx[0] - mn[0]) * (double)i / (double)nx;
                pts[3 * p + 1] = mn[1] + (mx[1] - mn[1]) * (double)j / (double)ny;
                pts[3 * p + 2] = mn[2] + (mx[2] - mn[2]) * (double)k / (double)nz;
            }
    /* faces registered cell by cell and deduplicated by their sorted vertex
     * key; the first registration owns the face (blockMesh.cpp:76-121) */
    const int64_t nReg = 6 * nx * ny * nz;
    face_ref* refs = (face_ref*)xcalloc((size_t)nReg, sizeof(face_ref));
    int64_t nRefs = 0;
    int64_t cap = 1;
    while (cap < 2 * nReg) cap <<= 1;
    int64_t* table = (int64_t*)xcalloc((size_t)cap, sizeof(int64_t));
    for (int64_t i = 0; i < cap; ++i) table[i] = -1;
    for (int64_t k = 0; k < nz; ++k)
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i)
            {
                const int64_t c = i + nx * (j + ny * k);
                const int64_t v0 = PAT(i, j, k), v1 = PAT(i + 1, j, k), v2 = PAT(i + 1, j + 1, k),
                              v3_ = PAT(i, j + 1, k), v4 = PAT(i, j, k + 1), v5 = PAT(i + 1, j, k + 1),
                              v6 = PAT(i + 1, j + 1, k + 1), v7 = PAT(i, j + 1, k + 1);
                const int64_t fl[6][4] = {{v0, v1, v2, v3_}, {v4, v5, v6, v7}, {v0, v1, v5, v4},
                                          {v2, v3_, v7, v6}, {v0, v3_, v7, v4}, {v1, v2, v6, v5}};
                for (int q = 0; q < 6; ++q)
                {
                    int64_t key[4];
                    sort4(fl[q], key);
                    uint64_t h = hash4(key) & (uint64_t)(cap - 1);
                    for (;;)
                    {
                        const int64_t e = table[h];
                        if (e < 0)
                        {
                            table[h] = nRefs;
                            face_ref* r = &refs[nRefs++];
                            memcpy(r->key, key, sizeof key);
                            memcpy(r->verts, fl[q], sizeof r->verts);
                            r->owner = c;
                            r->nbr = -1;
                            break;
                        }
                        if (memcmp(refs[e].key, key, sizeof key) == 0)
                        {
                            if (refs[e].nbr != -1) { free(refs); free(table); return fail("blockMesh: non-manifold face"); }
                            refs[e].nbr = c;
                            break;
                        }
                        h = (h + 1) & (uint64_t)(cap - 1);
                    }
                }
            }
#undef PAT
    free(table);
    /* internal faces in registration order, then boundary faces grouped by
     * side xmin xmax ymin ymax zmin zmax (blockMesh.cpp:123-185) */
    int64_t nf = 0, ni = 0;
    fOff[0] = 0;
    for (int64_t r = 0; r < nRefs; ++r)
    {
        face_ref* fr = &refs[r];
        if (fr->nbr == -1) continue;
        if (fr->owner > fr->nbr) { int64_t t = fr->owner; fr->owner = fr->nbr; fr->nbr = t; }
        for (int q = 0; q < 4; ++q) fV[4 * nf + q] = fr->verts[q];
        own[nf] = fr->owner;
        nbr[ni++] = fr->nbr;
        ++nf;
        fOff[nf] = 4 * nf;
    }
    int* side = (int*)xcalloc((size_t)nRefs, sizeof(int));
    for (int64_t r = 0; r < nRefs; ++r)
    {
        const face_ref* fr = &refs[r];
        if (fr->nbr != -1) continue;
        v3 cc = V3(0, 0, 0);
        for (int q = 0; q < 4; ++q) cc = vadd(cc, ld(pts, fr->verts[q]));
        cc = vdiv(cc, 4.0);
        const double eps = 1e-12;
        int s;
        if (fabs(cc.x - mn[0]) < eps) s = 0;
        else if (fabs(cc.x - mx[0]) < eps) s = 1;
        else if (fabs(cc.y - mn[1]) < eps) s = 2;
        else if (fabs(cc.y - mx[1]) < eps) s = 3;
        else if (fabs(cc.z - mn[2]) < eps) s = 4;
        else if (fabs(cc.z - mx[2]) < eps) s = 5;
        else { free(side); free(refs); return fail("blockMesh: boundary face not on any side"); }
        side[r] = s;
    }
    for (int s = 0; s < 6; ++s)
    {
        pStart[s] = nf;
        for (int64_t r = 0; r < nRefs; ++r)
        {
            const face_ref* fr = &refs[r];
            if (fr->nbr != -1 || side[r] != s) continue;
            for (int q = 0; q < 4; ++q) fV[4 * nf + q] = fr->verts[q];
            own[nf] = fr->owner;
            ++nf;
            fOff[nf] = 4 * nf;
        }
        pSize[s] = nf - pStart[s];
    }
    free(side);
    free(refs);
    if (nf != cnt[2] || ni != cnt[3]) return fail("blockMesh: face count mismatch");
    return 0;
}

/* ------------------------------------------------------------------------ */
/* polyMesh::calcGeometry (src/3d/src/mesh/polyMesh.cpp:83-288)             */
/* ------------------------------------------------------------------------ */

int cfo_geometry(cfo_mesh* m)
{
    const int64_t nF = m->nF, nC = m->nC, nInt = m->nInt;
    const double* P = m->pts;
    for (int64_t f = 0; f < nF; ++f)
    {
        const int64_t* vs = m->fV + m->fOff[f];
        const int64_t nv = m->fOff[f + 1] - m->fOff[f];
        const v3 v0 = ld(P, vs[0]);
        v3 n = V3(0, 0, 0);
        for (int64_t i = 1; i + 1 < nv; ++i)
            n = vadd(n, vcross(vsub(ld(P, vs[i]), v0), vsub(ld(P, vs[i + 1]), v0)));
        st(m->Sf, f, vmul(n, 0.5));
        int exactMean = nv == 3;
        if (nv == 4)
        {
            const v3 a = vadd(ld(P, vs[0]), ld(P, vs[2]));
            const v3 b = vadd(ld(P, vs[1]), ld(P, vs[3]));
            exactMean = a.x == b.x && a.y == b.y && a.z == b.z;
        }
        v3 c = V3(0, 0, 0);
        if (exactMean)
        {
            for (int64_t i = 0; i < nv; ++i) c = vadd(c, ld(P, vs[i]));
            st(m->Cf, f, vdiv(c, (double)nv));
        }
        else
        {
            const double wSum = vdot(n, n);
            if (wSum > 0)
            {
                for (int64_t i = 1; i + 1 < nv; ++i)
                {
                    const v3 vi = ld(P, vs[i]), vj = ld(P, vs[i + 1]);
                    const double w = vdot(vcross(vsub(vi, v0), vsub(vj, v0)), n);
                    c = vadd(c, vmul(vadd(vadd(v0, vi), vj), w));
                }
                st(m->Cf, f, vdiv(c, 3.0 * wSum));
            }
            else
            {
                for (int64_t i = 0; i < nv; ++i) c = vadd(c, ld(P, vs[i]));
                st(m->Cf, f, vdiv(c, (double)nv));
            }
        }
    }
    /* provisional centres from face-centre averages */
    double* est = (double*)xcalloc((size_t)(3 * nC), sizeof(double));
    int64_t* cnt = (int64_t*)xcalloc((size_t)nC, sizeof(int64_t));
    for (int64_t f = 0; f < nF; ++f)
    {
        const int64_t o = m->own[f];
        st(est, o, vadd(ld(est, o), ld(m->Cf, f)));
        ++cnt[o];
        if (f < nInt)
        {
            const int64_t nb = m->nbr[f];
            st(est, nb, vadd(ld(est, nb), ld(m->Cf, f)));
            ++cnt[nb];
        }
    }
    for (int64_t c = 0; c < nC; ++c)
        if (cnt[c] > 0) st(est, c, vdiv(ld(est, c), (double)cnt[c]));
    /* orientation with a relative tolerance */
    for (int64_t f = 0; f < nF; ++f)
    {
        const int64_t o = m->own[f];
        v3 dd;
        if (f < nInt) dd = vsub(ld(est, m->nbr[f]), ld(est, o));
        else dd = vsub(ld(m->Cf, f), ld(est, o));
        const v3 sf = ld(m->Sf, f);
        const double side = vdot(sf, dd);
        const double tol = 1e-12 * vmag(sf) * vmag(dd);
        if (side < -tol) st(m->Sf, f, vneg(sf));
    }
    for (int64_t f = 0; f < nF; ++f) m->magSf[f] = vmag(ld(m->Sf, f));
    /* divergence-theorem volumes and first moments */
    double* mom = (double*)xcalloc((size_t)(3 * nC), sizeof(double));
    for (int64_t c = 0; c < nC; ++c) m->V[c] = 0.0;
    for (int64_t f = 0; f < nF; ++f)
    {
        const int64_t* vs = m->fV + m->fOff[f];
        const int64_t nv = m->fOff[f + 1] - m->fOff[f];
        const v3 v0 = ld(P, vs[0]);
        double fv = 0;
        v3 fm = V3(0, 0, 0);
        for (int64_t i = 1; i + 1 < nv; ++i)
        {
            const v3 a = vsub(ld(P, vs[i]), v0);
            const v3 b = vsub(ld(P, vs[i + 1]), v0);
            const double tV = vdot(v0, vcross(a, b)) / 6.0;
            fv += tV;
            fm = vadd(fm, vmul(vdiv(vadd(vadd(v0, ld(P, vs[i])), ld(P, vs[i + 1])), 4.0), tV));
        }
        v3 raw = V3(0, 0, 0);
        for (int64_t i = 1; i + 1 < nv; ++i)
            raw = vadd(raw, vcross(vsub(ld(P, vs[i]), v0), vsub(ld(P, vs[i + 1]), v0)));
        const double s = vdot(raw, ld(m->Sf, f)) >= 0 ? 1.0 : -1.0;
        const int64_t o = m->own[f];
        m->V[o] += s * fv;
        st(mom, o, vadd(ld(mom, o), vmul(fm, s)));
        if (f < nInt)
        {
            const int64_t nb = m->nbr[f];
            m->V[nb] -= s * fv;
            st(mom, nb, vsub(ld(mom, nb), vmul(fm, s)));
        }
    }
    for (int64_t c = 0; c < nC; ++c)
    {
        st(m->C, c, vdiv(ld(mom, c), m->V[c]));
        m->V[c] = fabs(m->V[c]);
        if (m->V[c] <= 0)
        {
            free(est); free(cnt); free(mom);
            return fail("polyMesh: degenerate cell volume for cell %lld", (long long)c);
        }
    }
    for (int64_t f = 0; f < nF; ++f)
    {
        const int64_t o = m->own[f];
        v3 dv;
        if (f < nInt) dv = vsub(ld(m->C, m->nbr[f]), ld(m->C, o));
        else dv = vsub(ld(m->Cf, f), ld(m->C, o));
        st(m->d, f, dv);
        const double dm = vmag(dv);
        if (dm <= 0)
        {
            free(est); free(cnt); free(mom);
            return fail("polyMesh: zero owner-neighbour distance at face %lld", (long long)f);
        }
        m->invDist[f] = 1.0 / dm;
    }
    free(est);
    free(cnt);
    free(mom);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* interpolation weights (src/3d/src/discrete/interpolate.cpp:15-48)        */
/* ------------------------------------------------------------------------ */

void cfo_owner_weights(const cfo_mesh* m, double* ow)
{
    ow[0] = 0.5;
    for (int64_t f = 0; f < m->nInt; ++f)
    {
        const v3 dd = ld(m->d, f);
        const double d2 = vdot(dd, dd);
        const double nw = vdot(vsub(ld(m->Cf, f), ld(m->C, m->own[f])), dd) / d2;
        ow[f] = 1.0 - sclamp(nw, 0.0, 1.0);
    }
}

void cfo_skew(const cfo_mesh* m, const double* ow, double* skew)
{
    for (int64_t f = 0; f < m->nF; ++f) st(skew, f, V3(0, 0, 0));
    for (int64_t f = 0; f < m->nInt; ++f)
    {
        const v3 co = ld(m->C, m->own[f]), cn = ld(m->C, m->nbr[f]);
        const double nw = 1.0 - ow[f];
        st(skew, f, vsub(ld(m->Cf, f), vadd(co, vmul(vsub(cn, co), nw))));
    }
}

/* harmonicFaceGamma (src/3d/src/discrete/laplacianScheme.cpp:37-62) */
void cfo_harmonic_gamma(const cfo_mesh* m, double gamma, double* gf)
{
    for (int64_t f = 0; f < m->nF; ++f)
    {
        if (f < m->nInt)
        {
            const double gp = gamma, gn = gamma;
            const v3 cP = ld(m->C, m->own[f]), cN = ld(m->C, m->nbr[f]), cf = ld(m->Cf, f);
            const double dP = vmag(vsub(cf, cP)), dN = vmag(vsub(cN, cf));
            const double tot = dP + dN;
            gf[f] = (tot > 0 && gp > 0 && gn > 0) ? tot * gp * gn / (dN * gp + dP * gn) : 0.5 * (gp + gn);
        }
        else
        {
            gf[f] = gamma;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* gradients (src/3d/src/discrete/gradScheme.cpp)                           */
/* ------------------------------------------------------------------------ */

typedef struct
{
    const cfo_mesh* m;
    const double* ow;
    const double* skew;
} geo_ctx;

/* internal face value of the volScalarField overload (volFields.cpp:96-111):
 * the clamped owner-to-face fraction multiplies the OWNER value */
static double vol_face_value(const cfo_mesh* m, const double* data, int64_t f)
{
    const int64_t o = m->own[f];
    const v3 dd = ld(m->d, f);
    const double d2 = vdot(dd, dd);
    const double w = d2 > 0 ? smin(1.0, smax(0.0, vdot(vsub(ld(m->Cf, f), ld(m->C, o)), dd) / d2)) : 0.5;
    return w * data[o] + (1.0 - w) * data[m->nbr[f]];
}

/* gaussGrad (gradScheme.cpp:15-96).  bvals holds the boundary face values
 * faceValueOf(f, data) for f >= nInt. */
static void gauss_grad(const geo_ctx* g, const double* data, const double* bvals, int corrected,
                       int volQuirk, double* out)
{
    const cfo_mesh* m = g->m;
    const int64_t nC = m->nC, nF = m->nF, nInt = m->nInt;
    double* sum = (double*)xcalloc((size_t)(3 * nC), sizeof(double));
    double* gf = corrected ? (double*)xcalloc((size_t)(3 * nF), sizeof(double)) : NULL;
#define RECON(f)                                                                                   \
    ((corrected && (f) < nInt)                                                                     \
         ? g->ow[f] * data[m->own[f]] + (1.0 - g->ow[f]) * data[m->nbr[f]]                        \
         : ((f) < nInt ? (volQuirk ? vol_face_value(m, data, f)                                    \
                                   : g->ow[f] * data[m->own[f]] + (1.0 - g->ow[f]) * data[m->nbr[f]]) \
                       : bvals[(f) - nInt]))
    for (int64_t f = 0; f < nF; ++f)
    {
        const v3 flux = vmul(ld(m->Sf, f), RECON(f));
        st(sum, m->own[f], vadd(ld(sum, m->own[f]), flux));
        if (f < nInt) st(sum, m->nbr[f], vsub(ld(sum, m->nbr[f]), flux));
    }
    for (int64_t c = 0; c < nC; ++c) st(out, c, vdiv(ld(sum, c), m->V[c]));
    if (corrected)
    {
        for (int pass = 0; pass < 2; ++pass)
        {
            for (int64_t f = 0; f < nF; ++f)
            {
                if (f < nInt)
                {
                    const v3 gp = ld(out, m->own[f]), gn = ld(out, m->nbr[f]);
                    st(gf, f, vadd(vmul(gp, g->ow[f]), vmul(gn, 1.0 - g->ow[f])));
                }
                else
                {
                    st(gf, f, ld(out, m->own[f]));
                }
            }
            memset(sum, 0, sizeof(double) * (size_t)(3 * nC));
            for (int64_t f = 0; f < nF; ++f)
            {
                double tf = RECON(f);
                if (f < nInt) tf += vdot(ld(gf, f), ld(g->skew, f));
                const v3 flux = vmul(ld(m->Sf, f), tf);
                st(sum, m->own[f], vadd(ld(sum, m->own[f]), flux));
                if (f < nInt) st(sum, m->nbr[f], vsub(ld(sum, m->nbr[f]), flux));
            }
            for (int64_t c = 0; c < nC; ++c) st(out, c, vdiv(ld(sum, c), m->V[c]));
        }
    }
#undef RECON
    free(sum);
    free(gf);
}

/* Sym3 (gradScheme.cpp:106-137) */
typedef struct { double xx, xy, xz, yy, yz, zz; } sym3;

static void sym3_add(sym3* s, v3 d, double w)
{
    s->xx += w * d.x * d.x;
    s->xy += w * d.x * d.y;
    s->xz += w * d.x * d.z;
    s->yy += w * d.y * d.y;
    s->yz += w * d.y * d.z;
    s->zz += w * d.z * d.z;
}

static v3 sym3_solve(const sym3* s, v3 b)
{
    const double t = smax((s->xx + s->yy + s->zz) / 3.0, 1e-300);
    const double e = 1e-12 * t;
    const double XX = s->xx + e, YY = s->yy + e, ZZ = s->zz + e;
    const double c11 = YY * ZZ - s->yz * s->yz;
    const double c12 = s->xz * s->yz - s->xy * ZZ;
    const double c13 = s->xy * s->yz - YY * s->xz;
    const double c22 = XX * ZZ - s->xz * s->xz;
    const double c23 = s->xy * s->xz - XX * s->yz;
    const double c33 = XX * YY - s->xy * s->xy;
    const double det = XX * c11 + s->xy * c12 + s->xz * c13;
    if (det <= 0 || !isfinite(det)) return V3(0, 0, 0);
    return V3((c11 * b.x + c12 * b.y + c13 * b.z) / det, (c12 * b.x + c22 * b.y + c23 * b.z) / det,
              (c13 * b.x + c23 * b.y + c33 * b.z) / det);
}

/* leastSquaresGrad (gradScheme.cpp:154-239) */
static void ls_grad(const cfo_mesh* m, const double* data, const double* bvals, double* out)
{
    const int64_t nC = m->nC, nF = m->nF, nInt = m->nInt;
    sym3* cm = (sym3*)xcalloc((size_t)nC, sizeof(sym3));
    sym3* fmat = (sym3*)xcalloc((size_t)nC, sizeof(sym3));
    double* crhs = (double*)xcalloc((size_t)(3 * nC), sizeof(double));
    for (int64_t f = 0; f < nF; ++f)
    {
        const int64_t o = m->own[f];
        const v3 df = vsub(ld(m->Cf, f), ld(m->C, o));
        const double wf = 1.0 / smax(vmag(df), 1e-300);
        sym3_add(&fmat[o], df, wf);
        if (f < nInt)
        {
            const int64_t nb = m->nbr[f];
            const v3 dn = vsub(ld(m->C, nb), ld(m->C, o));
            const double wn = 1.0 / smax(vmag(dn), 1e-300);
            sym3_add(&cm[o], dn, wn);
            sym3_add(&cm[nb], dn, wn);
            const double dPhi = (data[nb] - data[o]) * wn;
            st(crhs, o, vadd(ld(crhs, o), vmul(dn, dPhi)));
            st(crhs, nb, vadd(ld(crhs, nb), vmul(dn, dPhi)));
            const v3 dfn = vsub(ld(m->Cf, f), ld(m->C, nb));
            sym3_add(&fmat[nb], dfn, 1.0 / smax(vmag(dfn), 1e-300));
        }
        else
        {
            sym3_add(&cm[o], df, wf);
            const double dPhi = (bvals[f - nInt] - data[o]) * wf;
            st(crhs, o, vadd(ld(crhs, o), vmul(df, dPhi)));
        }
    }
    double* g0 = (double*)xcalloc((size_t)(3 * nC), sizeof(double));
    for (int64_t c = 0; c < nC; ++c) st(g0, c, sym3_solve(&cm[c], ld(crhs, c)));
    double* frhs = crhs;
    memset(frhs, 0, sizeof(double) * (size_t)(3 * nC));
    for (int64_t f = 0; f < nF; ++f)
    {
        const int64_t o = m->own[f];
        double vf;
        if (f < nInt)
        {
            const int64_t nb = m->nbr[f];
            vf = 0.5 * ((data[o] + vdot(ld(g0, o), vsub(ld(m->Cf, f), ld(m->C, o))))
                        + (data[nb] + vdot(ld(g0, nb), vsub(ld(m->Cf, f), ld(m->C, nb)))));
            const v3 dN = vsub(ld(m->Cf, f), ld(m->C, nb));
            const double wN = 1.0 / smax(vmag(dN), 1e-300);
            st(frhs, nb, vadd(ld(frhs, nb), vmul(dN, (vf - data[nb]) * wN)));
        }
        else
        {
            vf = bvals[f - nInt];
        }
        const v3 dd = vsub(ld(m->Cf, f), ld(m->C, o));
        const double w = 1.0 / smax(vmag(dd), 1e-300);
        st(frhs, o, vadd(ld(frhs, o), vmul(dd, (vf - data[o]) * w)));
    }
    for (int64_t c = 0; c < nC; ++c) st(out, c, sym3_solve(&fmat[c], ld(frhs, c)));
    free(cm);
    free(fmat);
    free(crhs);
    free(g0);
}

static void grad_any(const geo_ctx* g, const double* data, const double* bvals, int scheme, int volQuirk,
                     double* out)
{
    if (scheme == CFO_GRAD_LEAST_SQUARES) ls_grad(g->m, data, bvals, out);
    else gauss_grad(g, data, bvals, scheme == CFO_GRAD_CORRECTED, volQuirk, out);
}

int cfo_grad(const cfo_mesh* m, const double* data, const double* bvals, int scheme, int volQuirk,
             double* out)
{
    double* ow = (double*)xcalloc((size_t)(m->nInt > 1 ? m->nInt : 1), sizeof(double));
    double* skew = (double*)xcalloc((size_t)(3 * m->nF), sizeof(double));
    cfo_owner_weights(m, ow);
    cfo_skew(m, ow, skew);
    geo_ctx g = {m, ow, skew};
    grad_any(&g, data, bvals, scheme, volQuirk, out);
    free(ow);
    free(skew);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* CSR and linear solvers (src/common/src/Matrix.cpp)                       */
/* ------------------------------------------------------------------------ */

static const int64_t* g_sortRows;
static const int64_t* g_sortCols;

static int trip_cmp(const void* a, const void* b)
{
    const int64_t i = *(const int64_t*)a, j = *(const int64_t*)b;
    if (g_sortRows[i] != g_sortRows[j]) return g_sortRows[i] < g_sortRows[j] ? -1 : 1;
    if (g_sortCols[i] != g_sortCols[j]) return g_sortCols[i] < g_sortCols[j] ? -1 : 1;
    return i < j ? -1 : (i > j);
}

/* finishWithDiagonal (Matrix.cpp:56-117): the triplets and one diagonal
 * triplet per row are sorted by (row, col) and duplicates summed.  Ties keep
 * insertion order here; the reference's sort is unstable, which only matters
 * for three or more duplicates (two summands commute exactly). */
int64_t cfo_csr_build(int64_t n, int64_t nTrip, const int64_t* rows, const int64_t* cols,
                      const double* vals, const double* diag, int64_t* rowStart, int64_t* outCols,
                      double* outVals)
{
    const int64_t tot = nTrip + (diag ? n : 0);
    int64_t* r = (int64_t*)xcalloc((size_t)tot, sizeof(int64_t));
    int64_t* c = (int64_t*)xcalloc((size_t)tot, sizeof(int64_t));
    double* v = (double*)xcalloc((size_t)tot, sizeof(double));
    int64_t* idx = (int64_t*)xcalloc((size_t)tot, sizeof(int64_t));
    memcpy(r, rows, sizeof(int64_t) * (size_t)nTrip);
    memcpy(c, cols, sizeof(int64_t) * (size_t)nTrip);
    memcpy(v, vals, sizeof(double) * (size_t)nTrip);
    if (diag)
        for (int64_t i = 0; i < n; ++i) { r[nTrip + i] = i; c[nTrip + i] = i; v[nTrip + i] = diag[i]; }
    for (int64_t k = 0; k < tot; ++k) idx[k] = k;
    g_sortRows = r;
    g_sortCols = c;
    qsort(idx, (size_t)tot, sizeof(int64_t), trip_cmp);
    for (int64_t i = 0; i <= n; ++i) rowStart[i] = 0;
    int64_t nnz = 0, prevRow = -1;
    for (int64_t k = 0; k < tot; ++k)
    {
        const int64_t rr = r[idx[k]], cc = c[idx[k]];
        const double vv = v[idx[k]];
        if (rr != prevRow)
        {
            for (int64_t q = prevRow + 1; q <= rr; ++q) rowStart[q] = nnz;
            outCols[nnz] = cc;
            outVals[nnz] = vv;
            ++nnz;
            prevRow = rr;
        }
        else if (outCols[nnz - 1] == cc)
        {
            outVals[nnz - 1] += vv;
        }
        else
        {
            outCols[nnz] = cc;
            outVals[nnz] = vv;
            ++nnz;
        }
    }
    for (int64_t q = prevRow + 1; q <= n; ++q) rowStart[q] = nnz;
    free(r);
    free(c);
    free(v);
    free(idx);
    return nnz;
}

void cfo_spmv(int64_t n, const int64_t* rs, const int64_t* cols, const double* vals, const double* x, double* y)
{
    for (int64_t r = 0; r < n; ++r)
    {
        double s = 0;
        for (int64_t k = rs[r]; k < rs[r + 1]; ++k) s += vals[k] * x[cols[k]];
        y[r] = s;
    }
}

static void csr_diag(int64_t n, const int64_t* rs, const int64_t* cols, const double* vals, double* d)
{
    for (int64_t r = 0; r < n; ++r)
    {
        d[r] = 0.0;
        for (int64_t k = rs[r]; k < rs[r + 1]; ++k)
            if (cols[k] == r) { d[r] = vals[k]; break; }
    }
}

static double sdot(int64_t n, const double* a, const double* b)
{
    double s = 0;
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

static double inf_norm(int64_t n, const double* v)
{
    double m = 0;
    for (int64_t i = 0; i < n; ++i)
    {
        if (isnan(v[i])) return NAN;
        m = smax(m, fabs(v[i]));
    }
    return m;
}

int cfo_solve_cg(int64_t n, const int64_t* rs, const int64_t* cols, const double* vals, const double* b,
                 double* x, double tol, int32_t maxIter, cfo_report* rep)
{
    double* d = (double*)xcalloc((size_t)n, sizeof(double));
    double* invD = (double*)xcalloc((size_t)n, sizeof(double));
    double* Ax = (double*)xcalloc((size_t)n, sizeof(double));
    double* r = (double*)xcalloc((size_t)n, sizeof(double));
    double* z = (double*)xcalloc((size_t)n, sizeof(double));
    double* p = (double*)xcalloc((size_t)n, sizeof(double));
    double* Ap = (double*)xcalloc((size_t)n, sizeof(double));
    csr_diag(n, rs, cols, vals, d);
    for (int64_t i = 0; i < n; ++i) invD[i] = (fabs(d[i]) > 1e-300) ? 1.0 / d[i] : 1.0;
    cfo_spmv(n, rs, cols, vals, x, Ax);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
    memset(rep, 0, sizeof *rep);
    rep->initialResidual = inf_norm(n, r);
    const double bnorm = smax(inf_norm(n, b), 1e-300);
    if (rep->initialResidual / bnorm < tol)
    {
        rep->converged = 1;
        rep->finalResidual = rep->initialResidual;
        goto done;
    }
    for (int64_t i = 0; i < n; ++i) z[i] = invD[i] * r[i];
    memcpy(p, z, sizeof(double) * (size_t)n);
    double rz = sdot(n, r, z);
    for (int it = 1; it <= maxIter; ++it)
    {
        cfo_spmv(n, rs, cols, vals, p, Ap);
        const double pAp = sdot(n, p, Ap);
        if (pAp <= 0 || fabs(rz) < 1e-300) break;
        const double alpha = rz / pAp;
        for (int64_t i = 0; i < n; ++i)
        {
            x[i] += alpha * p[i];
            r[i] -= alpha * Ap[i];
        }
        rep->iterations = it;
        rep->finalResidual = inf_norm(n, r);
        if (rep->finalResidual / bnorm < tol)
        {
            rep->converged = 1;
            break;
        }
        for (int64_t i = 0; i < n; ++i) z[i] = invD[i] * r[i];
        const double rzNew = sdot(n, r, z);
        const double beta = rzNew / rz;
        rz = rzNew;
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
done:
    free(d); free(invD); free(Ax); free(r); free(z); free(p); free(Ap);
    return 0;
}

int cfo_solve_bicgstab(int64_t n, const int64_t* rs, const int64_t* cols, const double* vals,
                       const double* b, double* x, double tol, int32_t maxIter, cfo_report* rep)
{
    double* d = (double*)xcalloc((size_t)n, sizeof(double));
    double* invD = (double*)xcalloc((size_t)n, sizeof(double));
    double* Ax = (double*)xcalloc((size_t)n, sizeof(double));
    double* r = (double*)xcalloc((size_t)n, sizeof(double));
    double* r0 = (double*)xcalloc((size_t)n, sizeof(double));
    double* p = (double*)xcalloc((size_t)n, sizeof(double));
    double* v = (double*)xcalloc((size_t)n, sizeof(double));
    double* s = (double*)xcalloc((size_t)n, sizeof(double));
    double* z = (double*)xcalloc((size_t)n, sizeof(double));
    double* sh = (double*)xcalloc((size_t)n, sizeof(double));
    double* t = (double*)xcalloc((size_t)n, sizeof(double));
    csr_diag(n, rs, cols, vals, d);
    for (int64_t i = 0; i < n; ++i) invD[i] = (d[i] > 1e-300) ? 1.0 / d[i] : 1.0;
    cfo_spmv(n, rs, cols, vals, x, Ax);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
    memset(rep, 0, sizeof *rep);
    rep->initialResidual = inf_norm(n, r);
    const double bnorm = smax(inf_norm(n, b), 1e-300);
    if (rep->initialResidual / bnorm < tol)
    {
        rep->converged = 1;
        rep->finalResidual = rep->initialResidual;
        goto done;
    }
    memcpy(r0, r, sizeof(double) * (size_t)n);
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    for (int it = 1; it <= maxIter; ++it)
    {
        const double rhoNew = sdot(n, r0, r);
        if (fabs(rhoNew) < 1e-300) break;
        const double beta = (rhoNew / rho) * (alpha / omega);
        rho = rhoNew;
        for (int64_t i = 0; i < n; ++i)
        {
            p[i] = r[i] + beta * (p[i] - omega * v[i]);
            z[i] = p[i] * invD[i];
        }
        cfo_spmv(n, rs, cols, vals, z, v);
        const double denom = sdot(n, r0, v);
        if (fabs(denom) < 1e-300) break;
        alpha = rho / denom;
        for (int64_t i = 0; i < n; ++i)
        {
            x[i] += alpha * z[i];
            s[i] = r[i] - alpha * v[i];
        }
        for (int64_t i = 0; i < n; ++i) sh[i] = s[i] * invD[i];
        cfo_spmv(n, rs, cols, vals, sh, t);
        const double tDenom = sdot(n, t, t);
        if (tDenom < 1e-300)
        {
            memcpy(r, s, sizeof(double) * (size_t)n);
            rep->iterations = it;
            rep->finalResidual = inf_norm(n, r);
            rep->converged = rep->finalResidual / bnorm < tol;
            break;
        }
        omega = sdot(n, t, s) / tDenom;
        for (int64_t i = 0; i < n; ++i)
        {
            x[i] += omega * sh[i];
            r[i] = s[i] - omega * t[i];
        }
        rep->iterations = it;
        rep->finalResidual = inf_norm(n, r);
        if (rep->finalResidual / bnorm < tol)
        {
            rep->converged = 1;
            break;
        }
    }
done:
    free(d); free(invD); free(Ax); free(r); free(r0); free(p); free(v); free(s); free(z); free(sh); free(t);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* boundary linearisation (src/3d/src/fields/volFields.cpp)                 */
/* ------------------------------------------------------------------------ */

typedef struct
{
    const cfo_mesh* m;
    int64_t* facePatch; /* nF, -1 internal */
} bc_ctx;

static double normal_distance(const cfo_mesh* m, int64_t f)
{
    const v3 sf = ld(m->Sf, f);
    const double a = vmag(sf);
    const v3 n = vdiv(sf, a);
    return vdot(ld(m->d, f), n);
}

static int dominant_axis(v3 n, int* axis)
{
    const double ax = fabs(n.x), ay = fabs(n.y), az = fabs(n.z);
    if (ax >= ay && ax >= az) { *axis = 0; return ax < 1.0 - 1e-6 ? -1 : 0; }
    if (ay >= az) { *axis = 1; return ay < 1.0 - 1e-6 ? -1 : 0; }
    *axis = 2;
    return az < 1.0 - 1e-6 ? -1 : 0;
}

/* volScalarField::linearise (volFields.cpp:117-147) */
static int lin_scalar(const cfo_mesh* m, int type, double value, int64_t f, double* c, double* k)
{
    switch (type)
    {
    case CFO_FIXED_VALUE: *c = 0; *k = value; return 0;
    case CFO_FIXED_GRADIENT: *c = 1; *k = value * normal_distance(m, f); return 0;
    case CFO_ZERO_GRADIENT:
    case CFO_SYMMETRY:
    case CFO_OUTLET: *c = 1; *k = 0; return 0;
    default: return fail("volScalarField: unknown patch bc type %d", type);
    }
}

/* volVectorField::linearise (volFields.cpp:246-283) */
static int lin_vector(const cfo_mesh* m, int type, v3 patchValue, const uint8_t* set, const double* fval,
                      int64_t f, int comp, double* c, double* k)
{
    const v3 value = (set && set[f]) ? ld(fval, f) : patchValue;
    switch (type)
    {
    case CFO_FIXED_VALUE: *c = 0; *k = vcomp(value, comp); return 0;
    case CFO_FIXED_GRADIENT: *c = 1; *k = vcomp(patchValue, comp) * normal_distance(m, f); return 0;
    case CFO_ZERO_GRADIENT:
    case CFO_OUTLET: *c = 1; *k = 0; return 0;
    case CFO_SYMMETRY:
    case CFO_WALL:
    {
        const v3 sf = ld(m->Sf, f);
        int ax;
        if (dominant_axis(vdiv(sf, vmag(sf)), &ax)) return fail("fields: symmetry normal not axis aligned");
        *c = (comp == ax) ? 0.0 : 1.0;
        *k = 0;
        return 0;
    }
    default: return fail("volVectorField: unknown patch bc type %d", type);
    }
}

/* ------------------------------------------------------------------------ */
/* fvMatrix (src/3d/src/discrete/fvMatrix.cpp) with the fvm terms           */
/* ------------------------------------------------------------------------ */

typedef struct
{
    int nComp;
    int64_t n;
    double* diag;  /* nComp*n */
    double* rhs;   /* nComp*n */
    double* x;     /* nComp*n */
    int64_t nTrip, capTrip;
    int64_t* tr;   /* per comp identical structure: shared row/col, per-comp values */
    int64_t* tc;
    double* tv;    /* nComp * capTrip */
    int preferCG;
    int useDIC; /* pressure: multicolour-DIC PCG instead of Jacobi */
    /* the laplacian corrector (laplacianScheme.cpp:217-263), if registered */
    int hasCorrector;
    double* corrGamma; /* nF */
    int corrSign;
    /* the unknown's boundary linearisation per comp and boundary face */
    double* bc_c;  /* nComp*(nF-nInt) */
    double* bc_k;
    /* CSR per comp */
    int64_t* rs;
    int64_t* cols;
    double* vals; /* nComp*nnz */
    int64_t nnz;
} fvmat;

static void fvmat_init(fvmat* e, int nComp, int64_t n, int64_t capTrip, int64_t nB)
{
    memset(e, 0, sizeof *e);
    e->nComp = nComp;
    e->n = n;
    e->diag = (double*)xcalloc((size_t)(nComp * n), sizeof(double));
    e->rhs = (double*)xcalloc((size_t)(nComp * n), sizeof(double));
    e->x = (double*)xcalloc((size_t)(nComp * n), sizeof(double));
    e->capTrip = capTrip;
    e->tr = (int64_t*)xcalloc((size_t)capTrip, sizeof(int64_t));
    e->tc = (int64_t*)xcalloc((size_t)capTrip, sizeof(int64_t));
    e->tv = (double*)xcalloc((size_t)(nComp * capTrip), sizeof(double));
    e->preferCG = 1;
    e->bc_c = (double*)xcalloc((size_t)(nComp * nB), sizeof(double));
    e->bc_k = (double*)xcalloc((size_t)(nComp * nB), sizeof(double));
}

static void fvmat_free(fvmat* e)
{
    free(e->diag); free(e->rhs); free(e->x); free(e->tr); free(e->tc); free(e->tv);
    free(e->bc_c); free(e->bc_k); free(e->rs); free(e->cols); free(e->vals); free(e->corrGamma);
}

/* one addOffDiag for every comp; comp values may differ */
static void add_off(fvmat* e, int64_t r, int64_t c, const double* vPerComp)
{
    const int64_t t = e->nTrip++;
    e->tr[t] = r;
    e->tc[t] = c;
    for (int q = 0; q < e->nComp; ++q) e->tv[q * e->capTrip + t] = vPerComp[q];
}

/* fvm::div (divScheme.cpp:11-62) */
static void fvm_div(fvmat* e, const geo_ctx* g, const double* phi, int scheme, double blendCoeff, int sign)
{
    const cfo_mesh* m = g->m;
    e->preferCG = 0;
    const double alpha = scheme == CFO_DIV_BLEND ? blendCoeff : (scheme == CFO_DIV_LINEAR ? 1.0 : 0.0);
    const int64_t nB = m->nF - m->nInt;
    for (int64_t f = 0; f < m->nF; ++f)
    {
        const int64_t o = m->own[f];
        const double p = phi[f];
        if (f < m->nInt)
        {
            const int64_t nb = m->nbr[f];
            double wPo = 0.0, wNo = 0.0;
            if (p >= 0) wPo = 1.0; else wNo = 1.0;
            if (alpha > 0)
            {
                const double c = g->ow[f];
                wPo = alpha * c + (1.0 - alpha) * wPo;
                wNo = alpha * (1.0 - c) + (1.0 - alpha) * wNo;
            }
            const double fp = (double)sign * p * wPo;
            const double fn = (double)sign * p * wNo;
            double vo[3], vn[3];
            for (int q = 0; q < e->nComp; ++q)
            {
                e->diag[q * e->n + o] += fp;
                vo[q] = fn;
                e->diag[q * e->n + nb] += -fn;
                vn[q] = -fp;
            }
            add_off(e, o, nb, vo);
            add_off(e, nb, o, vn);
        }
        else
        {
            for (int q = 0; q < e->nComp; ++q)
            {
                const double c = e->bc_c[q * nB + (f - m->nInt)], k = e->bc_k[q * nB + (f - m->nInt)];
                e->diag[q * e->n + o] += (double)sign * p * c;
                e->rhs[q * e->n + o] += (double)(-sign) * p * k;
            }
        }
    }
}

/* assembleLaplacian, static part (laplacianScheme.cpp:176-215) */
static void fvm_laplacian(fvmat* e, const geo_ctx* g, const double* gammaFace, int corrected, int sign)
{
    const cfo_mesh* m = g->m;
    const int64_t nB = m->nF - m->nInt;
    for (int64_t f = 0; f < m->nF; ++f)
    {
        const v3 dd = ld(m->d, f);
        const double d2 = vdot(dd, dd);
        const double oc = vdot(ld(m->Sf, f), dd) / d2;
        const double coef = gammaFace[f] * oc;
        const int64_t o = m->own[f];
        if (f < m->nInt)
        {
            const int64_t nb = m->nbr[f];
            double vv[3];
            for (int q = 0; q < e->nComp; ++q)
            {
                e->diag[q * e->n + o] += (double)(-sign) * coef;
                vv[q] = (double)sign * coef;
                e->diag[q * e->n + nb] += (double)(-sign) * coef;
            }
            add_off(e, o, nb, vv);
            add_off(e, nb, o, vv);
        }
        else
        {
            for (int q = 0; q < e->nComp; ++q)
            {
                const double c = e->bc_c[q * nB + (f - m->nInt)], k = e->bc_k[q * nB + (f - m->nInt)];
                e->diag[q * e->n + o] += (double)sign * coef * (c - 1.0);
                e->rhs[q * e->n + o] += (double)(-sign) * coef * k;
            }
        }
    }
    if (corrected)
    {
        e->hasCorrector = 1;
        e->corrSign = sign;
        e->corrGamma = (double*)xcalloc((size_t)m->nF, sizeof(double));
        memcpy(e->corrGamma, gammaFace, sizeof(double) * (size_t)m->nF);
    }
}

/* the corrector lambda (laplacianScheme.cpp:220-263) applied to x */
static void apply_corrector(fvmat* e, const geo_ctx* g, int gradScheme)
{
    const cfo_mesh* m = g->m;
    const int64_t nB = m->nF - m->nInt;
    double* gc = (double*)xcalloc((size_t)(3 * m->nC), sizeof(double));
    double* bv = (double*)xcalloc((size_t)nB, sizeof(double));
    const int sign = e->corrSign;
    for (int q = 0; q < e->nComp; ++q)
    {
        const double* xq = e->x + q * e->n;
        for (int64_t b = 0; b < nB; ++b)
            bv[b] = e->bc_c[q * nB + b] * xq[m->own[m->nInt + b]] + e->bc_k[q * nB + b];
        grad_any(g, xq, bv, gradScheme, 0, gc);
        for (int64_t f = 0; f < m->nF; ++f)
        {
            v3 gradFace;
            if (f < m->nInt)
                gradFace = vadd(vmul(ld(gc, m->own[f]), g->ow[f]), vmul(ld(gc, m->nbr[f]), 1.0 - g->ow[f]));
            else
                gradFace = ld(gc, m->own[f]);
            const v3 dd = ld(m->d, f);
            const double dm = vmag(dd);
            if (dm <= 0) continue;
            const v3 dh = vdiv(dd, dm);
            const v3 sfv = ld(m->Sf, f);
            const v3 cfVec = vsub(sfv, vmul(dh, vdot(sfv, dh)));
            const double corr = e->corrGamma[f] * vdot(cfVec, gradFace);
            e->rhs[q * e->n + m->own[f]] += (double)(-sign) * corr;
            if (f < m->nInt) e->rhs[q * e->n + m->nbr[f]] += (double)sign * corr;
        }
    }
    free(gc);
    free(bv);
}

static void fvmat_build_csr(fvmat* e)
{
    const int64_t n = e->n;
    const int64_t cap = e->nTrip + n;
    e->rs = (int64_t*)xcalloc((size_t)(n + 1), sizeof(int64_t));
    e->cols = (int64_t*)xcalloc((size_t)cap, sizeof(int64_t));
    e->vals = (double*)xcalloc((size_t)(e->nComp * cap), sizeof(double));
    for (int q = 0; q < e->nComp; ++q)
        e->nnz = cfo_csr_build(n, e->nTrip, e->tr, e->tc, e->tv + q * e->capTrip, e->diag + q * n, e->rs,
                               e->cols, e->vals + q * cap);
    /* compact per-comp value blocks to stride nnz */
    for (int q = 1; q < e->nComp; ++q)
        memmove(e->vals + q * e->nnz, e->vals + q * cap, sizeof(double) * (size_t)e->nnz);
}

/* fvMatrix::solve (fvMatrix.cpp:73-129), relaxation 1 */
static int64_t g_innerSum;
int cfo_solve_dic_cg(int64_t n, const int64_t* rs, const int64_t* cols, const double* vals, const double* b, double* x,
                     double tol, int32_t maxIter, cfo_report* rep);

static cfo_report fvmat_solve(fvmat* e, const geo_ctx* g, double tol, int maxIter, int nonOrth, int gradScheme)
{
    const int64_t n = e->n;
    double* base = (double*)xcalloc((size_t)(e->nComp * n), sizeof(double));
    memcpy(base, e->rhs, sizeof(double) * (size_t)(e->nComp * n));
    fvmat_build_csr(e);
    const int passes = !e->hasCorrector ? 1 : (nonOrth + 1 > 1 ? nonOrth + 1 : 1);
    cfo_report last;
    memset(&last, 0, sizeof last);
    for (int pass = 0; pass < passes; ++pass)
    {
        memcpy(e->rhs, base, sizeof(double) * (size_t)(e->nComp * n));
        if (e->hasCorrector) apply_corrector(e, g, gradScheme);
        for (int q = 0; q < e->nComp; ++q)
        {
            cfo_report rep;
            if (e->preferCG && e->useDIC)
                cfo_solve_dic_cg(n, e->rs, e->cols, e->vals + q * e->nnz, e->rhs + q * n, e->x + q * n, tol, maxIter,
                                 &rep);
            else if (e->preferCG)
                cfo_solve_cg(n, e->rs, e->cols, e->vals + q * e->nnz, e->rhs + q * n, e->x + q * n, tol, maxIter, &rep);
            else
                cfo_solve_bicgstab(n, e->rs, e->cols, e->vals + q * e->nnz, e->rhs + q * n, e->x + q * n, tol,
                                   maxIter, &rep);
            last = rep;
            g_innerSum += rep.iterations;
        }
    }
    free(base);
    return last;
}

/* fvMatrix::explicitOperator (fvMatrix.cpp:131-146) */
static void fvmat_h(const fvmat* e, const double* xIn, int comp, double* h)
{
    const int64_t n = e->n;
    double* ax = (double*)xcalloc((size_t)n, sizeof(double));
    cfo_spmv(n, e->rs, e->cols, e->vals + comp * e->nnz, xIn, ax);
    for (int64_t c = 0; c < n; ++c) h[c] = e->rhs[comp * n + c] - (ax[c] - e->diag[comp * n + c] * xIn[c]);
    free(ax);
}

/* ------------------------------------------------------------------------ */
/* SIMPLE (src/3d/src/solvers/simpleSolver.cpp:33-394)                      */
/* ------------------------------------------------------------------------ */

typedef struct
{
    geo_ctx g;
    double* ow;
    double* skew;
    int64_t* facePatch;
    double* gammaU;
    double* localScale;
} simple_ws;

static int ws_init(simple_ws* w, const cfo_mesh* m, double nu)
{
    memset(w, 0, sizeof *w);
    w->ow = (double*)xcalloc((size_t)(m->nInt > 1 ? m->nInt : 1), sizeof(double));
    w->skew = (double*)xcalloc((size_t)(3 * m->nF), sizeof(double));
    cfo_owner_weights(m, w->ow);
    cfo_skew(m, w->ow, w->skew);
    w->g.m = m;
    w->g.ow = w->ow;
    w->g.skew = w->skew;
    w->facePatch = (int64_t*)xcalloc((size_t)m->nF, sizeof(int64_t));
    for (int64_t f = 0; f < m->nF; ++f) w->facePatch[f] = -1;
    for (int64_t pi = 0; pi < m->nPatch; ++pi)
        for (int64_t f = m->pStart[pi]; f < m->pStart[pi] + m->pSize[pi]; ++f) w->facePatch[f] = pi;
    w->gammaU = (double*)xcalloc((size_t)m->nF, sizeof(double));
    cfo_harmonic_gamma(m, nu, w->gammaU);
    /* continuityError's per-cell largest face area (pressureCorrection.cpp:103-116) */
    w->localScale = (double*)xcalloc((size_t)m->nC, sizeof(double));
    for (int64_t f = 0; f < m->nF; ++f)
    {
        const double a = m->magSf[f];
        w->localScale[m->own[f]] = smax(w->localScale[m->own[f]], a);
        if (f < m->nInt) w->localScale[m->nbr[f]] = smax(w->localScale[m->nbr[f]], a);
    }
    return 0;
}

static void ws_free(simple_ws* w)
{
    free(w->ow); free(w->skew); free(w->facePatch); free(w->gammaU); free(w->localScale);
}

static void div_phi(const cfo_mesh* m, const double* phi, double* out)
{
    for (int64_t c = 0; c < m->nC; ++c) out[c] = 0.0;
    for (int64_t f = 0; f < m->nF; ++f)
    {
        out[m->own[f]] += phi[f];
        if (f < m->nInt) out[m->nbr[f]] -= phi[f];
    }
}

static double continuity_error(const cfo_mesh* m, const simple_ws* w, const double* phi)
{
    double* dv = (double*)xcalloc((size_t)m->nC, sizeof(double));
    div_phi(m, phi, dv);
    double err = 0;
    for (int64_t c = 0; c < m->nC; ++c) err = smax(err, fabs(dv[c]) / smax(w->localScale[c], 1e-300));
    free(dv);
    return err;
}

/* the U linearisation table for all boundary faces, comps 0..2 */
static int u_lin_table(const cfo_mesh* m, const simple_ws* w, const int32_t* types, const double* values,
                       const uint8_t* set, const double* fval, double* bc_c, double* bc_k)
{
    const int64_t nB = m->nF - m->nInt;
    for (int q = 0; q < 3; ++q)
        for (int64_t b = 0; b < nB; ++b)
        {
            const int64_t f = m->nInt + b;
            const int64_t pi = w->facePatch[f];
            if (lin_vector(m, types[pi], ld(values, pi), set, fval, f, q, &bc_c[q * nB + b], &bc_k[q * nB + b]))
                return -1;
        }
    return 0;
}

static int p_lin_table(const cfo_mesh* m, const simple_ws* w, const int32_t* types, const double* values,
                       double* bc_c, double* bc_k)
{
    const int64_t nB = m->nF - m->nInt;
    for (int64_t b = 0; b < nB; ++b)
    {
        const int64_t f = m->nInt + b;
        const int64_t pi = w->facePatch[f];
        if (lin_scalar(m, types[pi], values[pi], f, &bc_c[b], &bc_k[b])) return -1;
    }
    return 0;
}

/* fvc::grad of a volScalarField (gradScheme.cpp:246-261) */
static void vol_grad(const simple_ws* w, const double* data, const double* pc, const double* pk, int scheme,
                     double* out)
{
    const cfo_mesh* m = w->g.m;
    const int64_t nB = m->nF - m->nInt;
    double* bv = (double*)xcalloc((size_t)nB, sizeof(double));
    for (int64_t b = 0; b < nB; ++b) bv[b] = pc[b] * data[m->own[m->nInt + b]] + pk[b];
    grad_any(&w->g, data, bv, scheme, 1, out);
    free(bv);
}

/* correctFluxes (pressureCorrection.cpp:37-88) */
static void correct_fluxes(const simple_ws* w, const double* pCell, const double* pc, const double* pk,
                           const double* gradP, const double* rAUf, int corrected, double* phi)
{
    const cfo_mesh* m = w->g.m;
    for (int64_t f = 0; f < m->nF; ++f)
    {
        const v3 dcv = ld(m->d, f), sf = ld(m->Sf, f);
        const double d2 = vdot(dcv, dcv);
        if (d2 <= 0) continue;
        const double coef = rAUf[f] * vdot(sf, dcv) / d2;
        double corr = 0;
        if (corrected)
        {
            const v3 dh = vdiv(dcv, sqrt(d2));
            const v3 cfVec = vsub(sf, vmul(dh, vdot(sf, dh)));
            v3 gradFace;
            if (f < m->nInt)
                gradFace = vadd(vmul(ld(gradP, m->own[f]), w->ow[f]), vmul(ld(gradP, m->nbr[f]), 1.0 - w->ow[f]));
            else
                gradFace = ld(gradP, m->own[f]);
            corr = rAUf[f] * vdot(cfVec, gradFace);
        }
        if (f < m->nInt)
        {
            const double dp = pCell[m->nbr[f]] - pCell[m->own[f]];
            phi[f] -= coef * dp + corr;
        }
        else
        {
            const int64_t b = f - m->nInt;
            const double tp = pCell[m->own[f]];
            phi[f] -= coef * ((pc[b] - 1.0) * tp + pk[b]) + corr;
        }
    }
}

/* updatePhiInternal + correctBoundaryFlux for a vector field with a given
 * linearisation table (pressureCorrection.cpp:10-25, volFields.cpp:294-306) */
static void flux_from(const simple_ws* w, const double* Uc, const double* bc_c, const double* bc_k,
                      const int32_t* uTypes, double* phi)
{
    const cfo_mesh* m = w->g.m;
    const int64_t nB = m->nF - m->nInt;
    for (int64_t f = 0; f < m->nInt; ++f)
    {
        const v3 cO = ld(Uc, m->own[f]), cN = ld(Uc, m->nbr[f]);
        const v3 uf = vadd(vmul(cO, w->ow[f]), vmul(cN, 1.0 - w->ow[f]));
        phi[f] = vdot(uf, ld(m->Sf, f));
    }
    for (int64_t f = m->nInt; f < m->nF; ++f)
    {
        const int64_t b = f - m->nInt;
        if (uTypes[w->facePatch[f]] == CFO_EMPTY) { phi[f] = 0; continue; }
        const v3 tp = ld(Uc, m->own[f]);
        v3 out;
        for (int q = 0; q < 3; ++q) vset(&out, q, bc_c[q * nB + b] * vcomp(tp, q) + bc_k[q * nB + b]);
        phi[f] = vdot(out, ld(m->Sf, f));
    }
}

int cfo_flux_from_U(const cfo_mesh* m, const cfo_bcs* bc, const double* U, double* phi)
{
    simple_ws w;
    ws_init(&w, m, 1.0);
    const int64_t nB = m->nF - m->nInt;
    double* c = (double*)xcalloc((size_t)(3 * nB), sizeof(double));
    double* k = (double*)xcalloc((size_t)(3 * nB), sizeof(double));
    int rc = 0;
    if (u_lin_table(m, &w, bc->uType, bc->uValue, bc->uFaceSet, bc->uFaceValue, c, k)) rc = -1;
    else flux_from(&w, U, c, k, bc->uType, phi);
    free(c); free(k);
    ws_free(&w);
    return rc;
}

/* the momentum equation of one outer iteration (simpleSolver.cpp:67-112) */
/* Linear-upwind convection (this library's extension; the reference's
 * fvm::div knows upwind, linear and blend only, divScheme.cpp:18): the
 * face value is the upwind cell's value extrapolated along its gradient,
 * U_f = U_u + (grad U)_u . (Cf - C_u), u the upwind cell of phi_f >= 0 ->
 * owner.  The matrix keeps the upwind part; the extrapolation, evaluated on
 * the iterate the equation is assembled from with the gradient of each
 * component under U's conditions and the case's grad scheme, is a deferred
 * correction: -phi_f d_f on the owner's right-hand side, +phi_f d_f on the
 * neighbour's, summed per cell in face order and added after the other
 * right-hand-side terms.  The gradient interpolates internal faces with the
 * bounded owner weight (makeFaceValueFn, interpolate.cpp), as the
 * reference's strain rate of U does (turbulenceModel.cpp:197-211). */
static void linear_upwind_rhs(fvmat* U, const simple_ws* w, const cfo_controls* ctl, const double* uc,
                              const double* uk, const double* phi, const double* Ucur)
{
    const cfo_mesh* m = w->g.m;
    const int64_t nC = m->nC, nB = m->nF - m->nInt;
    double* comp = (double*)xcalloc((size_t)nC, sizeof(double));
    double* g = (double*)xcalloc((size_t)(3 * nC), sizeof(double));
    double* s = (double*)xcalloc((size_t)nC, sizeof(double));
    double* bv = (double*)xcalloc((size_t)nB + 1, sizeof(double));
    for (int q = 0; q < 3; ++q)
    {
        for (int64_t c = 0; c < nC; ++c) comp[c] = Ucur[3 * c + q];
        for (int64_t b = 0; b < nB; ++b) bv[b] = uc[q * nB + b] * comp[m->own[m->nInt + b]] + uk[q * nB + b];
        grad_any(&w->g, comp, bv, ctl->grad, 0, g);
        memset(s, 0, sizeof(double) * (size_t)nC);
        for (int64_t f = 0; f < m->nInt; ++f)
        {
            const int64_t o = m->own[f], nb = m->nbr[f];
            const double p = phi[f];
            const int64_t u = p >= 0 ? o : nb;
            const v3 d = vsub(ld(m->Cf, f), ld(m->C, u));
            const double corr = p * vdot(ld(g, u), d);
            s[o] = s[o] - corr;
            s[nb] = s[nb] + corr;
        }
        for (int64_t c = 0; c < nC; ++c) U->rhs[q * nC + c] += s[c];
    }
    free(comp);
    free(g);
    free(s);
    free(bv);
}

static int build_ueqn(fvmat* U, const simple_ws* w, const cfo_controls* ctl, const double* uc, const double* uk,
                      const double* phi, const double* gradPn, const double* Ucur)
{
    const cfo_mesh* m = w->g.m;
    const int64_t nB = m->nF - m->nInt;
    fvmat_init(U, 3, m->nC, 4 * m->nInt, nB);
    memcpy(U->bc_c, uc, sizeof(double) * (size_t)(3 * nB));
    memcpy(U->bc_k, uk, sizeof(double) * (size_t)(3 * nB));
    fvm_div(U, &w->g, phi, ctl->div == CFO_DIV_LINEAR_UPWIND ? CFO_DIV_UPWIND : ctl->div, ctl->blendCoeff, 1);
    fvm_laplacian(U, &w->g, w->gammaU, ctl->laplacianCorrected, -1);
    for (int64_t c = 0; c < m->nC; ++c)
    {
        const v3 f0 = V3(ctl->bodyForce[0], ctl->bodyForce[1], ctl->bodyForce[2]);
        const v3 rhs = vmul(vsub(vadd(f0, V3(0, 0, 0)), ld(gradPn, c)), m->V[c]);
        for (int q = 0; q < 3; ++q) U->rhs[q * m->nC + c] += vcomp(rhs, q);
    }
    if (ctl->div == CFO_DIV_LINEAR_UPWIND) linear_upwind_rhs(U, w, ctl, uc, uk, phi, Ucur);
    return 0;
}

static void build_peqn(fvmat* P, const simple_ws* w, const cfo_controls* ctl, const double* pc, const double* pk,
                       const double* rAUf, const double* dphi)
{
    const cfo_mesh* m = w->g.m;
    const int64_t nB = m->nF - m->nInt;
    fvmat_init(P, 1, m->nC, 2 * m->nInt, nB);
    memcpy(P->bc_c, pc, sizeof(double) * (size_t)nB);
    memcpy(P->bc_k, pk, sizeof(double) * (size_t)nB);
    fvm_laplacian(P, &w->g, rAUf, ctl->laplacianCorrected, -1);
    for (int64_t c = 0; c < m->nC; ++c) P->rhs[c] += -dphi[c];
    P->useDIC = ctl->pPrecond == 1;
    if (ctl->pRefCell >= 0 && ctl->pRefCell < m->nC)
    {
        const int64_t r = ctl->pRefCell;
        P->rhs[r] += P->diag[r] * ctl->pRefValue;
        P->diag[r] += P->diag[r];
    }
}

static void interp_to_faces(const simple_ws* w, const double* cell, double* face)
{
    const cfo_mesh* m = w->g.m;
    for (int64_t f = 0; f < m->nF; ++f)
    {
        if (f < m->nInt) face[f] = w->ow[f] * cell[m->own[f]] + (1.0 - w->ow[f]) * cell[m->nbr[f]];
        else face[f] = cell[m->own[f]];
    }
}

int cfo_simple(const cfo_mesh* m, const cfo_bcs* bc, const cfo_controls* ctl, double* U, double* p, double* phi,
               cfo_result* res)
{
    const int64_t nC = m->nC, nF = m->nF, nInt = m->nInt, nB = nF - nInt;
    memset(res, 0, sizeof *res);
    simple_ws w;
    ws_init(&w, m, ctl->nu);
    double* uc = (double*)xcalloc((size_t)(3 * nB), sizeof(double));
    double* uk = (double*)xcalloc((size_t)(3 * nB), sizeof(double));
    double* hc = (double*)xcalloc((size_t)(3 * nB), sizeof(double));
    double* hk = (double*)xcalloc((size_t)(3 * nB), sizeof(double));
    double* pc = (double*)xcalloc((size_t)nB, sizeof(double));
    double* pk = (double*)xcalloc((size_t)nB, sizeof(double));
    double* gradPn = (double*)xcalloc((size_t)(3 * nC), sizeof(double));
    double* gradPF = (double*)xcalloc((size_t)(3 * nC), sizeof(double));
    double* UOld = (double*)xcalloc((size_t)(3 * nC), sizeof(double));
    double* Hfree = (double*)xcalloc((size_t)(3 * nC), sizeof(double));
    double* rAUr = (double*)xcalloc((size_t)nC, sizeof(double));
    double* rAUf = (double*)xcalloc((size_t)nF, sizeof(double));
    double* dphi = (double*)xcalloc((size_t)nC, sizeof(double));
    double* pNew = (double*)xcalloc((size_t)nC, sizeof(double));
    int32_t* hTypes = (int32_t*)xcalloc((size_t)(m->nPatch ? m->nPatch : 1), sizeof(int32_t));
    double* hVals = (double*)xcalloc((size_t)(3 * (m->nPatch ? m->nPatch : 1)), sizeof(double));
    int rc = 0;
    if (u_lin_table(m, &w, bc->uType, bc->uValue, bc->uFaceSet, bc->uFaceValue, uc, uk)) { rc = -1; goto out; }
    if (p_lin_table(m, &w, bc->pType, bc->pValue, pc, pk)) { rc = -1; goto out; }
    /* constrainHbyA's boundary conditions (simpleSolver.cpp:175-187) */
    for (int64_t pi = 0; pi < m->nPatch; ++pi)
    {
        const int fixed = bc->uType[pi] == CFO_FIXED_VALUE;
        hTypes[pi] = fixed ? CFO_FIXED_VALUE : CFO_ZERO_GRADIENT;
        for (int q = 0; q < 3; ++q) hVals[3 * pi + q] = fixed ? bc->uValue[3 * pi + q] : 0.0;
    }
    if (u_lin_table(m, &w, hTypes, hVals, bc->uFaceSet, bc->uFaceValue, hc, hk)) { rc = -1; goto out; }
    int needReference = 1;
    for (int64_t pi = 0; pi < m->nPatch; ++pi)
        if (bc->pType[pi] == CFO_FIXED_VALUE) needReference = 0;

    double contLag1 = INFINITY, contLag2 = INFINITY;
    for (int iter = 1; iter <= ctl->maxIterations; ++iter)
    {
        vol_grad(&w, p, pc, pk, ctl->grad, gradPn);
        fvmat UE;
        build_ueqn(&UE, &w, ctl, uc, uk, phi, gradPn, U);
        g_innerSum = 0;
        const cfo_report uRep = fvmat_solve(&UE, &w.g, ctl->linearTol, ctl->linearMaxIter, ctl->nonOrthCorrectors, ctl->grad);
        res->uItersTotal += g_innerSum;
        res->lastUIters = uRep.iterations;
        memcpy(UOld, U, sizeof(double) * (size_t)(3 * nC));
        for (int q = 1; q < 3; ++q)
            for (int64_t c = 0; c < nC; ++c)
            {
                const double a = UE.diag[c], b = UE.diag[q * nC + c];
                if (fabs(a - b) > 1e-10 * (fabs(a) + fabs(b) + 1.0))
                {
                    fvmat_free(&UE);
                    rc = fail("SIMPLE: momentum diagonal differs between components");
                    goto out;
                }
            }
        for (int64_t c = 0; c < nC; ++c) rAUr[c] = m->V[c] / smax(UE.diag[c], 1e-300);
        for (int q = 0; q < 3; ++q)
            for (int64_t c = 0; c < nC; ++c)
                Hfree[3 * c + q] = (1.0 - ctl->relaxU) * UOld[3 * c + q] + ctl->relaxU * UE.x[q * nC + c];
        fvmat_free(&UE);
        flux_from(&w, Hfree, hc, hk, hTypes, phi);
        if (needReference)
        {
            double netSum = 0, freeSum = 0;
            for (int64_t pi = 0; pi < m->nPatch; ++pi)
            {
                const int fixedU = bc->uType[pi] == CFO_FIXED_VALUE;
                double s = 0;
                for (int64_t f = m->pStart[pi]; f < m->pStart[pi] + m->pSize[pi]; ++f) s += phi[f];
                netSum += s;
                if (!fixedU) freeSum += s;
            }
            if (fabs(freeSum) > 1e-30)
            {
                const double scale = (freeSum - netSum) / freeSum;
                for (int64_t pi = 0; pi < m->nPatch; ++pi)
                {
                    if (bc->uType[pi] == CFO_FIXED_VALUE) continue;
                    for (int64_t f = m->pStart[pi]; f < m->pStart[pi] + m->pSize[pi]; ++f) phi[f] *= scale;
                }
            }
        }
        const double contErr = continuity_error(m, &w, phi);
        div_phi(m, phi, dphi);
        interp_to_faces(&w, rAUr, rAUf);
        fvmat PE;
        build_peqn(&PE, &w, ctl, pc, pk, rAUf, dphi);
        g_innerSum = 0;
        const cfo_report pRep = fvmat_solve(&PE, &w.g, ctl->linearTol, ctl->linearMaxIter, ctl->nonOrthCorrectors, ctl->grad);
        res->pItersTotal += g_innerSum;
        res->lastPIters = pRep.iterations;
        memcpy(pNew, PE.x, sizeof(double) * (size_t)nC);
        fvmat_free(&PE);
        vol_grad(&w, pNew, pc, pk, ctl->grad, gradPF);
        correct_fluxes(&w, pNew, pc, pk, gradPF, rAUf, ctl->laplacianCorrected, phi);
        double pStep = 0, pScale = 0;
        for (int64_t c = 0; c < nC; ++c)
        {
            pStep = smax(pStep, fabs(pNew[c] - p[c]));
            pScale = smax(pScale, fabs(p[c]));
        }
        const double aP = ctl->pRelaxStart > 0
                              ? smin(ctl->relaxP, smax(ctl->pRelaxStart, 0.15 * pScale / smax(pStep, 1e-300)))
                              : ctl->relaxP;
        double pDeltaMax = 0;
        for (int64_t c = 0; c < nC; ++c)
        {
            const double dp = aP * (pNew[c] - p[c]);
            pDeltaMax = smax(pDeltaMax, fabs(dp));
            p[c] += dp;
            const double s = aP * rAUr[c];
            const v3 corr = vmul(vsub(ld(gradPF, c), ld(gradPn, c)), s);
            st(U, c, vsub(ld(Hfree, c), corr));
        }
        const double errAfter = continuity_error(m, &w, phi);
        double uMax = 0, dUMax = 0;
        int finite = 1;
        for (int64_t c = 0; c < nC; ++c)
        {
            uMax = smax(uMax, vmag(ld(U, c)));
            dUMax = smax(dUMax, vmag(vsub(ld(U, c), ld(UOld, c))));
            if (!isfinite(U[3 * c]) || !isfinite(U[3 * c + 1]) || !isfinite(U[3 * c + 2]) || !isfinite(p[c])) finite = 0;
        }
        const double uRes = dUMax / smax(uMax, 1e-300);
        if (ctl->verbose)
            printf("[cfo] SIMPLE iter %d: continuity %g (corrected %g, dp %g, dU %g)\n", iter, contErr, errAfter,
                   pDeltaMax, uRes);
        res->iterations = iter;
        res->finalContinuityError = contErr;
        res->finalMomentumResidual = uRes;
        if (!isfinite(contErr) || !isfinite(pDeltaMax) || !finite) break;
        const int settled = contErr <= contLag2 * 1.01 + 1e-12;
        const int momentumSettled = !(ctl->momentumTol > 0) || uRes <= ctl->momentumTol;
        if (momentumSettled &&
            (contErr < ctl->continuityTol || (iter >= 5 && ctl->pcorrTol > 0 && pDeltaMax < ctl->pcorrTol && settled)))
        {
            res->converged = 1;
            break;
        }
        contLag2 = contLag1;
        contLag1 = contErr;
    }
out:
    free(uc); free(uk); free(hc); free(hk); free(pc); free(pk); free(gradPn); free(gradPF); free(UOld);
    free(Hfree); free(rAUr); free(rAUf); free(dphi); free(pNew); free(hTypes); free(hVals);
    ws_free(&w);
    res->error = rc;
    return rc;
}

int cfo_eqns(const cfo_mesh* m, const cfo_bcs* bc, const cfo_controls* ctl, const double* U, const double* p,
             const double* phi, const double* xprobe, double* gradPn, double* uDiag, double* uH0, double* uH1,
             double* rAUf, double* divPhiOut, double* contErr, double* pDiag, double* pH0, double* pH1,
             double* gradPFull, double* phiCorrected)
{
    (void)U;
    const int64_t nC = m->nC, nF = m->nF, nB = m->nF - m->nInt;
    simple_ws w;
    ws_init(&w, m, ctl->nu);
    double* uc = (double*)xcalloc((size_t)(3 * nB), sizeof(double));
    double* uk = (double*)xcalloc((size_t)(3 * nB), sizeof(double));
    double* pc = (double*)xcalloc((size_t)nB, sizeof(double));
    double* pk = (double*)xcalloc((size_t)nB, sizeof(double));
    double* zero = (double*)xcalloc((size_t)nC, sizeof(double));
    double* rAUr = (double*)xcalloc((size_t)nC, sizeof(double));
    int rc = 0;
    if (u_lin_table(m, &w, bc->uType, bc->uValue, bc->uFaceSet, bc->uFaceValue, uc, uk) ||
        p_lin_table(m, &w, bc->pType, bc->pValue, pc, pk))
    {
        rc = -1;
        goto out;
    }
    vol_grad(&w, p, pc, pk, ctl->grad, gradPn);
    fvmat UE;
    build_ueqn(&UE, &w, ctl, uc, uk, phi, gradPn, U);
    fvmat_solve(&UE, &w.g, ctl->linearTol, 0, 0, ctl->grad);
    for (int q = 0; q < 3; ++q)
    {
        memcpy(uDiag + q * nC, UE.diag + q * nC, sizeof(double) * (size_t)nC);
        fvmat_h(&UE, zero, q, uH0 + q * nC);
        fvmat_h(&UE, xprobe, q, uH1 + q * nC);
    }
    for (int64_t c = 0; c < nC; ++c) rAUr[c] = m->V[c] / smax(UE.diag[c], 1e-300);
    fvmat_free(&UE);
    interp_to_faces(&w, rAUr, rAUf);
    div_phi(m, phi, divPhiOut);
    *contErr = continuity_error(m, &w, phi);
    fvmat PE;
    build_peqn(&PE, &w, ctl, pc, pk, rAUf, divPhiOut);
    fvmat_solve(&PE, &w.g, ctl->linearTol, 0, 0, ctl->grad);
    memcpy(pDiag, PE.diag, sizeof(double) * (size_t)nC);
    fvmat_h(&PE, zero, 0, pH0);
    fvmat_h(&PE, xprobe, 0, pH1);
    fvmat_free(&PE);
    vol_grad(&w, xprobe, pc, pk, ctl->grad, gradPFull);
    memcpy(phiCorrected, phi, sizeof(double) * (size_t)nF);
    correct_fluxes(&w, xprobe, pc, pk, gradPFull, rAUf, ctl->laplacianCorrected, phiCorrected);
out:
    free(uc); free(uk); free(pc); free(pk); free(zero); free(rAUr);
    ws_free(&w);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Multicolour DIC preconditioner (no reference counterpart; the reference's */
/* "DICG" stand-in is Jacobi, src/common/include/cf/common/Matrix.h:65-72).  */
/* Restates the definition chuanflow_b200 implements so its device result   */
/* can be checked bit-for-bit:                                               */
/*   colours: greedy first-fit over cells in ascending order, the smallest   */
/*            colour not used by an already-coloured neighbour;              */
/*   lower(i): off-diagonal entries of row i whose column has a smaller      */
/*            colour, in ascending column order; upper(i) likewise larger;   */
/*   factor:  colour by colour ascending, rD_i = ((a_ii - t_1) - t_2) ...,   */
/*            t_k = a_ij^2 / rD_j over lower(i), stored as 1 / rD_i;         */
/*   apply:   forward colour by colour, z_i = rDinv_i (r_i - sum a_ij z_j)   */
/*            over lower(i); backward colours descending (all but the last), */
/*            z_i = z_i - rDinv_i (sum a_ij z_j) over upper(i).              */
/* ------------------------------------------------------------------------ */

int cfo_colour_cells(int64_t n, const int64_t* rs, const int64_t* cols, int32_t* colour)
{
    int32_t* mark = (int32_t*)xcalloc((size_t)(n + 2), sizeof(int32_t));
    for (int64_t i = 0; i < n; ++i) colour[i] = -1;
    int32_t nColours = 0;
    for (int64_t i = 0; i < n; ++i)
    {
        for (int64_t k = rs[i]; k < rs[i + 1]; ++k)
        {
            const int64_t j = cols[k];
            if (j != i && colour[j] >= 0) mark[colour[j]] = (int32_t)(i + 1);
        }
        int32_t c = 0;
        while (mark[c] == (int32_t)(i + 1)) ++c;
        colour[i] = c;
        if (c + 1 > nColours) nColours = c + 1;
    }
    free(mark);
    return nColours;
}

int cfo_dic_factor(int64_t n, const int64_t* rs, const int64_t* cols, const double* vals, const int32_t* colour,
                   int32_t nColours, double* rDinv)
{
    double* rD = (double*)xcalloc((size_t)n, sizeof(double));
    for (int32_t c = 0; c < nColours; ++c)
        for (int64_t i = 0; i < n; ++i)
        {
            if (colour[i] != c) continue;
            double d = 0;
            for (int64_t k = rs[i]; k < rs[i + 1]; ++k)
                if (cols[k] == i) { d = vals[k]; break; }
            for (int64_t k = rs[i]; k < rs[i + 1]; ++k)
            {
                const int64_t j = cols[k];
                if (j != i && colour[j] < c) d = d - vals[k] * vals[k] / rD[j];
            }
            rD[i] = d;
            rDinv[i] = 1.0 / d;
        }
    free(rD);
    return 0;
}

void cfo_dic_apply(int64_t n, const int64_t* rs, const int64_t* cols, const double* vals, const int32_t* colour,
                   int32_t nColours, const double* rDinv, const double* r, double* z)
{
    for (int32_t c = 0; c < nColours; ++c)
        for (int64_t i = 0; i < n; ++i)
        {
            if (colour[i] != c) continue;
            double s = 0;
            for (int64_t k = rs[i]; k < rs[i + 1]; ++k)
            {
                const int64_t j = cols[k];
                if (j != i && colour[j] < c) s += vals[k] * z[j];
            }
            z[i] = rDinv[i] * (r[i] - s);
        }
    for (int32_t c = nColours - 2; c >= 0; --c)
        for (int64_t i = 0; i < n; ++i)
        {
            if (colour[i] != c) continue;
            double s = 0;
            for (int64_t k = rs[i]; k < rs[i + 1]; ++k)
            {
                const int64_t j = cols[k];
                if (j != i && colour[j] > c) s += vals[k] * z[j];
            }
            z[i] = z[i] - rDinv[i] * s;
        }
}

/* PCG of Matrix.cpp:153-222 with z = M^-1 r from the multicolour DIC */
int cfo_solve_dic_cg(int64_t n, const int64_t* rs, const int64_t* cols, const double* vals, const double* b, double* x,
                     double tol, int32_t maxIter, cfo_report* rep)
{
    int32_t* colour = (int32_t*)xcalloc((size_t)n, sizeof(int32_t));
    const int32_t nc = cfo_colour_cells(n, rs, cols, colour);
    double* rDinv = (double*)xcalloc((size_t)n, sizeof(double));
    cfo_dic_factor(n, rs, cols, vals, colour, nc, rDinv);
    double* Ax = (double*)xcalloc((size_t)n, sizeof(double));
    double* r = (double*)xcalloc((size_t)n, sizeof(double));
    double* z = (double*)xcalloc((size_t)n, sizeof(double));
    double* p = (double*)xcalloc((size_t)n, sizeof(double));
    double* Ap = (double*)xcalloc((size_t)n, sizeof(double));
    cfo_spmv(n, rs, cols, vals, x, Ax);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
    memset(rep, 0, sizeof *rep);
    rep->initialResidual = inf_norm(n, r);
    const double bnorm = smax(inf_norm(n, b), 1e-300);
    if (rep->initialResidual / bnorm < tol)
    {
        rep->converged = 1;
        rep->finalResidual = rep->initialResidual;
        goto done;
    }
    cfo_dic_apply(n, rs, cols, vals, colour, nc, rDinv, r, z);
    memcpy(p, z, sizeof(double) * (size_t)n);
    double rz = sdot(n, r, z);
    for (int it = 1; it <= maxIter; ++it)
    {
        cfo_spmv(n, rs, cols, vals, p, Ap);
        const double pAp = sdot(n, p, Ap);
        if (pAp <= 0 || fabs(rz) < 1e-300) break;
        const double alpha = rz / pAp;
        for (int64_t i = 0; i < n; ++i)
        {
            x[i] += alpha * p[i];
            r[i] -= alpha * Ap[i];
        }
        rep->iterations = it;
        rep->finalResidual = inf_norm(n, r);
        if (rep->finalResidual / bnorm < tol)
        {
            rep->converged = 1;
            break;
        }
        cfo_dic_apply(n, rs, cols, vals, colour, nc, rDinv, r, z);
        const double rzNew = sdot(n, r, z);
        const double beta = rzNew / rz;
        rz = rzNew;
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
done:
    free(colour); free(rDinv); free(Ax); free(r); free(z); free(p); free(Ap);
    return 0;
}

/* The pressure matrix of one outer iteration for a given rAUf: the static
 * part of fvm::laplacianFace (laplacianScheme.cpp:176-215, sign -1) with the
 * optional reference cell, as CSR (Matrix.cpp:56-117).  rs: nC+1, cols and
 * vals: room for nC + 2 nInt entries; returns nnz. */
int64_t cfo_pressure_csr(const cfo_mesh* m, const cfo_bcs* bc, const cfo_controls* ctl, const double* rAUf,
                         int64_t* rs, int64_t* cols, double* vals)
{
    simple_ws w;
    ws_init(&w, m, ctl->nu);
    const int64_t nB = m->nF - m->nInt;
    double* pc = (double*)xcalloc((size_t)nB, sizeof(double));
    double* pk = (double*)xcalloc((size_t)nB, sizeof(double));
    double* zero = (double*)xcalloc((size_t)m->nC, sizeof(double));
    int64_t nnz = -1;
    if (p_lin_table(m, &w, bc->pType, bc->pValue, pc, pk) == 0)
    {
        fvmat P;
        build_peqn(&P, &w, ctl, pc, pk, rAUf, zero);
        fvmat_build_csr(&P);
        nnz = P.nnz;
        memcpy(rs, P.rs, sizeof(int64_t) * (size_t)(m->nC + 1));
        memcpy(cols, P.cols, sizeof(int64_t) * (size_t)nnz);
        memcpy(vals, P.vals, sizeof(double) * (size_t)nnz);
        fvmat_free(&P);
    }
    free(pc); free(pk); free(zero);
    ws_free(&w);
    return nnz;
}

/* ------------------------------------------------------------------------
 * Device cell numbering (the library's cellOrder, no reference counterpart):
 * restated here so the permutation is checked element for element.
 *   adjacency: distinct neighbours across internal faces, ascending;
 *   colours:   first fit in ascending cell order (cfo_colour_cells);
 *   RCM:       per component, root = unnumbered cell of least (degree,
 *              index), moved at most 8 times to the least-(degree, index)
 *              cell of its farthest BFS level while the eccentricity grows;
 *              breadth-first numbering with neighbours by (degree, index);
 *              the whole sequence reversed;
 *   modes:     0 identity, 1 colour blocks of the identity, 2 RCM,
 *              3 colour blocks of the RCM order (stable).
 * ------------------------------------------------------------------------ */
static const int64_t* g_ord_deg;

static int ord_less(int64_t a, int64_t b)
{
    return g_ord_deg[a] != g_ord_deg[b] ? g_ord_deg[a] < g_ord_deg[b] : a < b;
}

static int ord_cmp(const void* pa, const void* pb)
{
    const int64_t a = *(const int64_t*)pa, b = *(const int64_t*)pb;
    return ord_less(a, b) ? -1 : (ord_less(b, a) ? 1 : 0);
}

static int i64_cmp(const void* pa, const void* pb)
{
    const int64_t a = *(const int64_t*)pa, b = *(const int64_t*)pb;
    return a < b ? -1 : (a > b ? 1 : 0);
}

/* BFS levels from root over unnumbered cells; eccentricity returned, the
 * farthest level left in last[0..*nLast) */
static int ord_bfs(int64_t nC, const int64_t* rs, const int64_t* adj, int64_t root, const char* numbered,
                   int64_t* stamp, int64_t tag, int64_t* last, int64_t* nLast, int64_t* buf)
{
    int64_t* cur = buf;
    int64_t* next = buf + nC;
    int64_t nCur = 1, nNext;
    cur[0] = root;
    stamp[root] = tag;
    int ecc = 0;
    for (;;)
    {
        nNext = 0;
        for (int64_t a = 0; a < nCur; ++a)
        {
            const int64_t u = cur[a];
            for (int64_t k = rs[u]; k < rs[u + 1]; ++k)
            {
                const int64_t v = adj[k];
                if (numbered[v] || stamp[v] == tag) continue;
                stamp[v] = tag;
                next[nNext++] = v;
            }
        }
        if (nNext == 0) break;
        int64_t* t = cur;
        cur = next;
        next = t;
        nCur = nNext;
        ++ecc;
    }
    memcpy(last, cur, (size_t)nCur * sizeof(int64_t));
    *nLast = nCur;
    return ecc;
}

int cfo_cell_order(int64_t nC, int64_t nInt, const int64_t* own, const int64_t* nbr, int32_t mode,
                   int64_t* newToOld)
{
    for (int64_t c = 0; c < nC; ++c) newToOld[c] = c;
    if (mode == 0) return 0;
    int64_t* rs = (int64_t*)xcalloc((size_t)(nC + 1), sizeof(int64_t));
    for (int64_t f = 0; f < nInt; ++f)
    {
        ++rs[own[f] + 1];
        ++rs[nbr[f] + 1];
    }
    for (int64_t c = 0; c < nC; ++c) rs[c + 1] += rs[c];
    int64_t* fill = (int64_t*)xcalloc((size_t)nC + 1, sizeof(int64_t));
    int64_t* adj = (int64_t*)xcalloc((size_t)rs[nC] + 1, sizeof(int64_t));
    for (int64_t c = 0; c < nC; ++c) fill[c] = rs[c];
    for (int64_t f = 0; f < nInt; ++f)
    {
        adj[fill[own[f]]++] = nbr[f];
        adj[fill[nbr[f]]++] = own[f];
    }
    int64_t w = 0, s0 = 0;
    for (int64_t c = 0; c < nC; ++c)
    {
        const int64_t b = s0, e = rs[c + 1];
        qsort(adj + b, (size_t)(e - b), sizeof(int64_t), i64_cmp);
        for (int64_t k = b; k < e; ++k)
            if (k == b || adj[k] != adj[k - 1]) adj[w++] = adj[k];
        s0 = e;
        rs[c + 1] = w;
    }
    if (mode == 2 || mode == 3)
    {
        int64_t* deg = (int64_t*)xcalloc((size_t)nC + 1, sizeof(int64_t));
        for (int64_t c = 0; c < nC; ++c) deg[c] = rs[c + 1] - rs[c];
        g_ord_deg = deg;
        int64_t* byDeg = (int64_t*)xcalloc((size_t)nC + 1, sizeof(int64_t));
        for (int64_t c = 0; c < nC; ++c) byDeg[c] = c;
        qsort(byDeg, (size_t)nC, sizeof(int64_t), ord_cmp);
        char* numbered = (char*)xcalloc((size_t)nC + 1, 1);
        int64_t* stamp = (int64_t*)xcalloc((size_t)nC + 1, sizeof(int64_t));
        for (int64_t c = 0; c < nC; ++c) stamp[c] = -1;
        int64_t* last = (int64_t*)xcalloc((size_t)nC + 1, sizeof(int64_t));
        int64_t* last2 = (int64_t*)xcalloc((size_t)nC + 1, sizeof(int64_t));
        int64_t* buf = (int64_t*)xcalloc((size_t)(2 * nC) + 2, sizeof(int64_t));
        int64_t* nb = (int64_t*)xcalloc((size_t)nC + 1, sizeof(int64_t));
        int64_t* order = (int64_t*)xcalloc((size_t)nC + 1, sizeof(int64_t));
        int64_t nOrd = 0, scan = 0, tag = 0, nLast = 0, nLast2 = 0;
        while (nOrd < nC)
        {
            while (numbered[byDeg[scan]]) ++scan;
            int64_t root = byDeg[scan];
            int ecc = ord_bfs(nC, rs, adj, root, numbered, stamp, tag++, last, &nLast, buf);
            for (int round = 0; round < 8; ++round)
            {
                int64_t cand = last[0];
                for (int64_t a = 0; a < nLast; ++a)
                    if (ord_less(last[a], cand)) cand = last[a];
                const int ecc2 = ord_bfs(nC, rs, adj, cand, numbered, stamp, tag++, last2, &nLast2, buf);
                if (ecc2 <= ecc) break;
                root = cand;
                ecc = ecc2;
                memcpy(last, last2, (size_t)nLast2 * sizeof(int64_t));
                nLast = nLast2;
            }
            int64_t head = nOrd;
            order[nOrd++] = root;
            numbered[root] = 1;
            while (head < nOrd)
            {
                const int64_t u = order[head++];
                int64_t m = 0;
                for (int64_t k = rs[u]; k < rs[u + 1]; ++k)
                    if (!numbered[adj[k]]) nb[m++] = adj[k];
                qsort(nb, (size_t)m, sizeof(int64_t), ord_cmp);
                for (int64_t a = 0; a < m; ++a)
                {
                    numbered[nb[a]] = 1;
                    order[nOrd++] = nb[a];
                }
            }
        }
        for (int64_t i = 0; i < nC; ++i) newToOld[i] = order[nC - 1 - i];
        free(deg);
        free(byDeg);
        free(numbered);
        free(stamp);
        free(last);
        free(last2);
        free(buf);
        free(nb);
        free(order);
    }
    if (mode == 1 || mode == 3)
    {
        int32_t* colour = (int32_t*)xcalloc((size_t)nC + 1, sizeof(int32_t));
        const int32_t nCol = cfo_colour_cells(nC, rs, adj, colour);
        int64_t* tmp = (int64_t*)xcalloc((size_t)nC + 1, sizeof(int64_t));
        int64_t t = 0;
        for (int32_t col = 0; col < nCol; ++col)
            for (int64_t i = 0; i < nC; ++i)
                if (colour[newToOld[i]] == col) tmp[t++] = newToOld[i];
        memcpy(newToOld, tmp, (size_t)nC * sizeof(int64_t));
        free(colour);
        free(tmp);
    }
    free(rs);
    free(fill);
    free(adj);
    return 0;
}
