// The extern "C" boundary: status codes, the per-thread error message, and
// the case-file runner.
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>

#include "cfg_internal.h"
#include "ctx.h"
#include "dict.h"

namespace
{

thread_local std::string g_lastError;

template <class F>
int guard(F&& f)
{
    try
    {
        f();
        return CFG_OK;
    }
    catch (const cfg::Error& e)
    {
        g_lastError = e.what();
        return e.code;
    }
    catch (const std::bad_alloc&)
    {
        g_lastError = "out of host memory";
        return CFG_ENOMEM;
    }
    catch (const std::exception& e)
    {
        g_lastError = e.what();
        return CFG_EINVAL;
    }
}

void need(bool ok, const char* what)
{
    if (!ok) cfg::fail(CFG_EINVAL, what);
}

int bcFromName(const std::string& s)
{
    if (s == "fixedValue") return CFG_BC_FIXED_VALUE;
    if (s == "zeroGradient") return CFG_BC_ZERO_GRADIENT;
    if (s == "fixedGradient") return CFG_BC_FIXED_GRADIENT;
    if (s == "symmetry") return CFG_BC_SYMMETRY;
    if (s == "outlet") return CFG_BC_OUTLET;
    if (s == "wall") return CFG_BC_WALL;
    if (s == "empty") return CFG_BC_EMPTY;
    cfg::fail(CFG_ESETUP, "unknown patch bc type '" + s + "'");
}

uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ULL;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

}  // namespace

namespace cfg
{
void setLastError(const std::string& msg) { g_lastError = msg; }
}  // namespace cfg

extern "C" {

size_t cfg_last_error(char* buf, size_t size)
{
    if (buf && size)
    {
        const size_t n = std::min(size - 1, g_lastError.size());
        std::memcpy(buf, g_lastError.data(), n);
        buf[n] = 0;
    }
    return g_lastError.size();
}

const char* cfg_version(void) { return "chuanflow_b200 0.1"; }

int cfg_mesh_create(const double* points, int64_t nP, const int64_t* faceOffsets, const int64_t* faceVerts,
                    int64_t nF, const int64_t* owner, const int64_t* neighbour, int64_t nInt, int32_t nPatch,
                    const char* const* names, const char* const* types, const int64_t* pStart,
                    const int64_t* pSize, cfg_mesh** out)
{
    return guard([&] {
        need(out && points && faceOffsets && faceVerts && owner && nP > 0 && nF > 0, "cfg_mesh_create: null argument");
        need(nInt >= 0 && nInt <= nF && (nInt == 0 || neighbour), "cfg_mesh_create: bad internal face count");
        auto m = std::make_unique<cfg_mesh>();
        m->m.points.resize(nP);
        for (int64_t i = 0; i < nP; ++i) m->m.points[i] = {points[3 * i], points[3 * i + 1], points[3 * i + 2]};
        m->m.faceOffsets.assign(faceOffsets, faceOffsets + nF + 1);
        need(faceOffsets[0] == 0, "cfg_mesh_create: face_offsets[0] must be 0");
        m->m.faceVerts.assign(faceVerts, faceVerts + faceOffsets[nF]);
        m->m.owner.assign(owner, owner + nF);
        m->m.neighbour.assign(neighbour, neighbour + nInt);
        for (int32_t i = 0; i < nPatch; ++i)
        {
            cfg::Mesh::Patch p;
            p.name = names && names[i] ? names[i] : "patch" + std::to_string(i);
            p.type = types && types[i] ? types[i] : "wall";
            p.start = pStart[i];
            p.size = pSize[i];
            m->m.patches.push_back(p);
        }
        m->m.finish();
        *out = m.release();
    });
}

int cfg_mesh_block(const double mn[3], const double mx[3], int64_t nx, int64_t ny, int64_t nz,
                   const char* const* sideNames, const char* const* sideTypes, cfg_mesh** out)
{
    return guard([&] {
        need(out && mn && mx, "cfg_mesh_block: null argument");
        // BlockSides defaults (src/3d/include/cf/fvm/BlockMesh.h:13-21)
        std::vector<std::string> names = {"xmin", "xmax", "ymin", "ymax", "zmin", "zmax"};
        std::vector<std::string> types = {"wall", "wall", "wall", "wall", "symmetry", "symmetry"};
        for (int s = 0; s < 6; ++s)
        {
            if (sideNames && sideNames[s]) names[s] = sideNames[s];
            if (sideTypes && sideTypes[s]) types[s] = sideTypes[s];
        }
        auto m = std::make_unique<cfg_mesh>();
        m->m = cfg::blockMesh({mn[0], mn[1], mn[2]}, {mx[0], mx[1], mx[2]}, nx, ny, nz, names, types);
        *out = m.release();
    });
}

int cfg_mesh_from_cells(const double* points, int64_t nP, const int32_t* types, const int64_t* cellOffsets,
                        const int64_t* cellVerts, int64_t nCells, cfg_mesh** out)
{
    return guard([&] {
        need(out && points && types && cellOffsets && cellVerts && nP > 0 && nCells > 0,
             "cfg_mesh_from_cells: null argument");
        std::vector<cfg::Vec> pts(static_cast<size_t>(nP));
        for (int64_t i = 0; i < nP; ++i) pts[i] = {points[3 * i], points[3 * i + 1], points[3 * i + 2]};
        std::vector<int32_t> ty(types, types + nCells);
        std::vector<int64_t> off(cellOffsets, cellOffsets + nCells + 1);
        need(off[0] == 0, "cfg_mesh_from_cells: cell_offsets[0] must be 0");
        std::vector<int64_t> cv(cellVerts, cellVerts + off[nCells]);
        for (int64_t v : cv) need(v >= 0 && v < nP, "cfg_mesh_from_cells: vertex index out of range");
        auto m = std::make_unique<cfg_mesh>();
        m->m = cfg::meshFromCells(pts, ty, off, cv);
        *out = m.release();
    });
}

int cfg_mesh_read_gmsh(const char* path, int32_t nTypes, const char* const* names, const char* const* types,
                       cfg_mesh** out)
{
    return guard([&] {
        need(path && out && (nTypes == 0 || (names && types)), "cfg_mesh_read_gmsh: null argument");
        std::map<std::string, std::string> pt;
        for (int32_t i = 0; i < nTypes; ++i) pt[names[i]] = types[i];
        auto m = std::make_unique<cfg_mesh>();
        m->m = cfg::readGmsh(path, pt);
        *out = m.release();
    });
}

int cfg_mesh_move_points(cfg_mesh* mesh, const double* points, int64_t nP)
{
    return guard([&] {
        need(mesh && points, "cfg_mesh_move_points: null argument");
        if (nP != static_cast<int64_t>(mesh->m.points.size()))
            cfg::fail(CFG_EMESH, "polyMesh::movePoints: point count changed; topology is fixed in ALE");
        for (int64_t i = 0; i < nP; ++i) mesh->m.points[i] = {points[3 * i], points[3 * i + 1], points[3 * i + 2]};
        mesh->m.calcGeometry();
    });
}

int cfg_mesh_jitter_interior(cfg_mesh* mesh, double fraction, uint64_t seed)
{
    return guard([&] {
        need(mesh, "cfg_mesh_jitter_interior: null mesh");
        cfg::Mesh& M = mesh->m;
        if (M.bnx < 0) cfg::fail(CFG_EINVAL, "cfg_mesh_jitter_interior: mesh did not come from a block");
        const int64_t nx = M.bnx, ny = M.bny, nz = M.bnz;
        const double h[3] = {(M.bmax.x - M.bmin.x) / static_cast<double>(nx),
                             (M.bmax.y - M.bmin.y) / static_cast<double>(ny),
                             (M.bmax.z - M.bmin.z) / static_cast<double>(nz)};
        const uint64_t s0 = seed * 0x100000001B3ULL;
        for (int64_t k = 1; k < nz; ++k)
            for (int64_t j = 1; j < ny; ++j)
                for (int64_t i = 1; i < nx; ++i)
                {
                    const int64_t pidx = i + (nx + 1) * (j + (ny + 1) * k);
                    double* c[3] = {&M.points[pidx].x, &M.points[pidx].y, &M.points[pidx].z};
                    for (int a = 0; a < 3; ++a)
                    {
                        const uint64_t r = splitmix64(s0 ^ (static_cast<uint64_t>(pidx) * 3ULL + static_cast<uint64_t>(a)));
                        const double u = static_cast<double>(r >> 11) * (1.0 / 9007199254740992.0);
                        *c[a] += (u * 2.0 - 1.0) * fraction * h[a];
                    }
                }
        M.calcGeometry();
    });
}

void cfg_mesh_destroy(cfg_mesh* mesh) { delete mesh; }

int cfg_mesh_counts(const cfg_mesh* mesh, int64_t counts[5])
{
    return guard([&] {
        need(mesh && counts, "cfg_mesh_counts: null argument");
        counts[0] = static_cast<int64_t>(mesh->m.points.size());
        counts[1] = mesh->m.nCells;
        counts[2] = mesh->m.nFaces();
        counts[3] = mesh->m.nInternal();
        counts[4] = static_cast<int64_t>(mesh->m.patches.size());
    });
}

int cfg_mesh_patch(const cfg_mesh* mesh, int32_t patch, char* name, size_t nameSize, char* type, size_t typeSize,
                   int64_t* start, int64_t* size)
{
    return guard([&] {
        need(mesh && patch >= 0 && patch < static_cast<int32_t>(mesh->m.patches.size()), "cfg_mesh_patch: bad patch");
        const auto& p = mesh->m.patches[patch];
        if (name && nameSize) std::snprintf(name, nameSize, "%s", p.name.c_str());
        if (type && typeSize) std::snprintf(type, typeSize, "%s", p.type.c_str());
        if (start) *start = p.start;
        if (size) *size = p.size;
    });
}

int cfg_mesh_patch_id(const cfg_mesh* mesh, const char* name)
{
    if (!mesh || !name) return -1;
    for (size_t i = 0; i < mesh->m.patches.size(); ++i)
        if (mesh->m.patches[i].name == name) return static_cast<int>(i);
    g_lastError = std::string("polyMesh: no patch named '") + name + "'";
    return -1;
}

int cfg_mesh_addressing(const cfg_mesh* mesh, double* points, int64_t* faceOffsets, int64_t* faceVerts,
                        int64_t* owner, int64_t* neighbour)
{
    return guard([&] {
        need(mesh != nullptr, "cfg_mesh_addressing: null mesh");
        const cfg::Mesh& M = mesh->m;
        if (points)
            for (size_t i = 0; i < M.points.size(); ++i)
            {
                points[3 * i] = M.points[i].x;
                points[3 * i + 1] = M.points[i].y;
                points[3 * i + 2] = M.points[i].z;
            }
        if (faceOffsets) std::memcpy(faceOffsets, M.faceOffsets.data(), M.faceOffsets.size() * sizeof(int64_t));
        if (faceVerts) std::memcpy(faceVerts, M.faceVerts.data(), M.faceVerts.size() * sizeof(int64_t));
        if (owner) std::memcpy(owner, M.owner.data(), M.owner.size() * sizeof(int64_t));
        if (neighbour && !M.neighbour.empty()) std::memcpy(neighbour, M.neighbour.data(), M.neighbour.size() * sizeof(int64_t));
    });
}

int cfg_mesh_geometry(const cfg_mesh* mesh, double* V, double* C, double* Cf, double* Sf, double* magSf, double* d,
                      double* invDist)
{
    return guard([&] {
        need(mesh != nullptr, "cfg_mesh_geometry: null mesh");
        const cfg::Mesh& M = mesh->m;
        auto vec = [](double* out, const std::vector<cfg::Vec>& v) {
            if (!out) return;
            for (size_t i = 0; i < v.size(); ++i)
            {
                out[3 * i] = v[i].x;
                out[3 * i + 1] = v[i].y;
                out[3 * i + 2] = v[i].z;
            }
        };
        if (V) std::memcpy(V, M.V.data(), M.V.size() * sizeof(double));
        vec(C, M.C);
        vec(Cf, M.Cf);
        vec(Sf, M.Sf);
        if (magSf) std::memcpy(magSf, M.magSf.data(), M.magSf.size() * sizeof(double));
        vec(d, M.d);
        if (invDist) std::memcpy(invDist, M.invDist.data(), M.invDist.size() * sizeof(double));
    });
}

int cfg_mesh_weights(const cfg_mesh* mesh, double* ow, double* skew)
{
    return guard([&] {
        need(mesh != nullptr, "cfg_mesh_weights: null mesh");
        const auto w = mesh->m.ownerWeights();
        if (ow) std::memcpy(ow, w.data(), w.size() * sizeof(double));
        if (skew)
        {
            const auto s = mesh->m.skewVectors(w);
            for (size_t i = 0; i < s.size(); ++i)
            {
                skew[3 * i] = s[i].x;
                skew[3 * i + 1] = s[i].y;
                skew[3 * i + 2] = s[i].z;
            }
        }
    });
}

int cfg_mesh_device_order(const cfg_mesh* mesh, int32_t order, int64_t* newToOld)
{
    return guard([&] {
        need(mesh && newToOld, "cfg_mesh_device_order: null argument");
        const std::vector<int64_t> o = cfg::cellOrder(mesh->m, order);
        std::copy(o.begin(), o.end(), newToOld);
    });
}

int cfg_ctx_create_ordered(const cfg_mesh* mesh, int32_t device, void* stream, int32_t order, cfg_ctx** out)
{
    return guard([&] {
        need(mesh && out, "cfg_ctx_create: null argument");
        auto c = std::make_unique<cfg_ctx>();
        c->c = std::make_unique<cfg::Ctx>(mesh->m, device, static_cast<cudaStream_t>(stream), order);
        *out = c.release();
    });
}

int cfg_ctx_create(const cfg_mesh* mesh, int32_t device, void* stream, cfg_ctx** out)
{
    return cfg_ctx_create_ordered(mesh, device, stream, CFG_ORDER_DEFAULT, out);
}

void cfg_ctx_destroy(cfg_ctx* ctx) { delete ctx; }

int cfg_set_patch_bc(cfg_ctx* ctx, char field, int32_t patch, int32_t type, const double* value)
{
    return guard([&] {
        need(ctx != nullptr, "cfg_set_patch_bc: null context");
        ctx->c->setPatchBC(field, patch, type, value);
    });
}

int cfg_set_face_values_U(cfg_ctx* ctx, int64_t n, const int64_t* faces, const double* values)
{
    return guard([&] {
        need(ctx && (n == 0 || (faces && values)), "cfg_set_face_values_U: null argument");
        ctx->c->setFaceValuesU(n, faces, values);
    });
}

int cfg_clear_face_values_U(cfg_ctx* ctx)
{
    return guard([&] {
        need(ctx != nullptr, "null context");
        ctx->c->clearFaceValuesU();
    });
}

int cfg_set_schemes(cfg_ctx* ctx, const cfg_schemes* s)
{
    return guard([&] {
        need(ctx && s, "cfg_set_schemes: null argument");
        need(s->div >= 0 && s->div <= CFG_DIV_LINEAR_UPWIND && s->grad >= 0 && s->grad <= 2, "cfg_set_schemes: unknown scheme");
        ctx->c->setSchemes(*s);
    });
}

int cfg_fields_upload(cfg_ctx* ctx, const double* U, const double* p, const double* phi)
{
    return guard([&] {
        need(ctx != nullptr, "null context");
        ctx->c->upload(U, p, phi);
    });
}

int cfg_fields_upload_old(cfg_ctx* ctx, const double* U_old)
{
    return guard([&] {
        need(ctx && U_old, "cfg_fields_upload_old: null argument");
        ctx->c->uploadOld(U_old);
    });
}

int cfg_fields_download(cfg_ctx* ctx, double* U, double* p, double* phi)
{
    return guard([&] {
        need(ctx != nullptr, "null context");
        ctx->c->download(U, p, phi);
    });
}

int cfg_fields_init_flux(cfg_ctx* ctx, const double* u0)
{
    return guard([&] {
        need(ctx != nullptr, "null context");
        ctx->c->initFlux(u0);
    });
}

int cfg_simple_iterate(cfg_ctx* ctx, const cfg_simple_controls* ctl, cfg_simple_result* res)
{
    return guard([&] {
        need(ctx && ctl && res, "cfg_simple_iterate: null argument");
        need(ctl->linear_max_iter >= 0 && ctl->max_iterations >= 0, "cfg_simple_iterate: negative iteration limit");
        ctx->c->iterate(*ctl, *res);
    });
}

int cfg_last_timing(const cfg_ctx* ctx, double ms[8], int64_t* launches)
{
    return guard([&] {
        need(ctx && ms, "cfg_last_timing: null argument");
        for (int i = 0; i < 8; ++i) ms[i] = ctx->c->lastMs[i];
        if (launches) *launches = ctx->c->lastLaunches;
    });
}

int cfg_kernel_timing(cfg_ctx* ctx, int32_t enable)
{
    return guard([&] {
        need(ctx != nullptr, "null context");
        ctx->c->setKernelTiming(enable != 0);
    });
}

static_assert(cfg::Ctx::KS_COUNT == CFG_KERNEL_SLOTS, "the header's slot count");

int cfg_kernel_stats(const cfg_ctx* ctx, double* out, int32_t slots)
{
    return guard([&] {
        need(ctx && out, "cfg_kernel_stats: null argument");
        need(slots >= 0, "cfg_kernel_stats: negative slot count");
        for (int k = 0; k < cfg::Ctx::KS_COUNT && k < slots; ++k)
        {
            out[2 * k] = ctx->c->kstat[k][0];
            out[2 * k + 1] = ctx->c->kstat[k][1];
        }
    });
}

int cfg_kernel_components(const cfg_ctx* ctx, double* out, int32_t slots)
{
    return guard([&] {
        need(ctx && out, "cfg_kernel_components: null argument");
        need(slots >= 0, "cfg_kernel_components: negative slot count");
        for (int k = 0; k < cfg::Ctx::KS_COUNT && k < slots; ++k) out[k] = ctx->c->kcomp[k];
    });
}

int cfg_sparse_solve(const cfg_ctx* ctx, int32_t device, int64_t n, const int64_t* rs, const int64_t* cols,
                     const double* vals, const double* b, double* x, double tol, int32_t maxIter, int32_t method,
                     cfg_solver_report* rep)
{
    (void)ctx;
    return guard([&] {
        need(rs && cols && vals && b && x && rep, "cfg_sparse_solve: null argument");
        need(method == CFG_SOLVE_CG || method == CFG_SOLVE_BICGSTAB, "cfg_sparse_solve: unknown method");
        cfg::Ctx::sparseSolve(device, n, rs, cols, vals, b, x, tol, maxIter, method, rep);
    });
}

/* test diagnostics (not part of the reference surface) */
int cfg_probe_equations(cfg_ctx* ctx, const cfg_simple_controls* ctl, const double* xprobe, double* out)
{
    return guard([&] {
        need(ctx && ctl && xprobe && out, "cfg_probe_equations: null argument");
        ctx->c->probeEquations(*ctl, xprobe, out);
    });
}

int cfg_probe_dic(cfg_ctx* ctx, const double* r, double* z, double* rdinv, int32_t* n_colours)
{
    return guard([&] {
        need(ctx && r && z && rdinv, "cfg_probe_dic: null argument");
        ctx->c->probeDIC(r, z, rdinv);
        if (n_colours) *n_colours = ctx->c->nColours();
    });
}

int cfg_poisson_setup(cfg_ctx* ctx, int64_t ref_cell)
{
    return guard([&] {
        need(ctx != nullptr, "cfg_poisson_setup: null context");
        ctx->c->poissonSetup(ref_cell);
    });
}

int cfg_poisson_solve(cfg_ctx* ctx, const double* b, double* x, int32_t method, double rel_tol, int32_t max_iter,
                      int32_t inner_max_iter, double inner_rel_tol, cfg_poisson_report* report)
{
    return guard([&] {
        need(ctx && b && x && report, "cfg_poisson_solve: null argument");
        double out[6];
        ctx->c->poissonSolve(b, x, method, rel_tol, max_iter, inner_max_iter, inner_rel_tol, out);
        report->inner_iterations = static_cast<int64_t>(out[0]);
        report->outer_iterations = static_cast<int32_t>(out[1]);
        report->converged = static_cast<int32_t>(out[2]);
        report->true_rel_residual = out[3];
        report->device_ms = out[4];
        report->initial_rel_residual = out[5];
    });
}

int cfg_poisson_amg_setup(cfg_ctx* ctx, double out[11])
{
    return guard([&] {
        need(ctx && out, "cfg_poisson_amg_setup: null argument");
        ctx->c->poissonAmg(out);
    });
}

int cfg_poisson_amg_apply(cfg_ctx* ctx, const double* r, double* z)
{
    return guard([&] {
        need(ctx && r && z, "cfg_poisson_amg_apply: null argument");
        ctx->c->poissonAmgApply(r, z);
    });
}

int cfg_poisson_amg_apply3(cfg_ctx* ctx, const double* r, double* z, const int32_t done[3])
{
    return guard([&] {
        need(ctx && r && z && done, "cfg_poisson_amg_apply3: null argument");
        ctx->c->poissonAmgApply3(r, z, done);
    });
}

int cfg_amg_strength(cfg_ctx* ctx, double theta)
{
    return guard([&] {
        need(ctx, "cfg_amg_strength: null argument");
        ctx->c->setAmgStrength(theta);
    });
}

int cfg_gradient(cfg_ctx* ctx, const double* data, const double* bvals, int32_t scheme, int32_t volQuirk, double* out)
{
    return guard([&] {
        need(ctx && data && bvals && out, "cfg_gradient: null argument");
        ctx->c->gradient(data, bvals, scheme, volQuirk, out);
    });
}

}  // extern "C"

namespace
{

/// A chflow-simple-foam case parsed on the host: mesh, boundary conditions
/// (per patch: U type/value, p type/value), initial U, schemes, controls.
struct CaseSpec
{
    cfg::Mesh mesh;
    std::vector<int> uType, pType;
    std::vector<std::array<double, 3>> uVal;
    std::vector<double> pVal;
    bool hasU0 = false;
    double u0[3] = {0, 0, 0};
    cfg_schemes schemes{CFG_DIV_UPWIND, 1, CFG_GRAD_CORRECTED, 0.9};
    cfg_simple_controls ctl{};
    // turbulence{} (TurbulenceConfig, TurbulenceModel.h:50-59 defaults)
    std::string turbModel = "laminar";
    double turbIntensity = 0.05, turbLength = -1, turbRelax = 0.7;
    double cDES = 0.61, reOnset = 0, onsetWidth = -1, gammaRate = 4.0;
};

CaseSpec parseCase(const char* path)
{
    const cfg::Dict d = cfg::Dict::parseFile(path);
    CaseSpec cs;
    // mesh: block{} (BlockMesh::fromDict, blockMesh.cpp:191-223) or mesh{} of a
    // gmsh file (meshLoader.cpp:14-59)
    const bool hasBlock = d.has("block"), hasFile = d.has("mesh");
    if (hasBlock && hasFile) cfg::fail(CFG_ESETUP, "case: block {} and mesh {} are mutually exclusive");
    if (!hasBlock && !hasFile) cfg::fail(CFG_ESETUP, "case: no mesh; add a block {} or a mesh {} section");
    if (hasFile)
    {
        const cfg::Dict& md = d.dict("mesh");
        const std::string format = md.wordOr("format", "gmsh");
        if (format != "gmsh") cfg::fail(CFG_ESETUP, "mesh: format '" + format + "' is unknown (gmsh is supported)");
        std::string file = md.word("file");
        if (!file.empty() && file[0] != '/')
        {
            // a relative file not found from the working directory is looked
            // up beside the case dictionary
            std::FILE* probe = std::fopen(file.c_str(), "rb");
            if (probe) std::fclose(probe);
            else
            {
                const std::string dir(path);
                const size_t slash = dir.find_last_of('/');
                if (slash != std::string::npos)
                {
                    const std::string beside = dir.substr(0, slash + 1) + file;
                    std::FILE* p2 = std::fopen(beside.c_str(), "rb");
                    if (p2)
                    {
                        std::fclose(p2);
                        file = beside;
                    }
                }
            }
        }
        std::map<std::string, std::string> patchTypes;
        if (md.has("patches"))
        {
            const cfg::Dict& ps = md.dict("patches");
            for (const auto& name : ps.keys()) patchTypes[name] = ps.dict(name).wordOr("type", "wall");
        }
        cs.mesh = cfg::readGmsh(file, patchTypes);
    }
    else
    {
    const cfg::Dict& b = d.dict("block");
    const auto mn = b.numbers("min"), mx = b.numbers("max"), nc = b.numbers("cells");
    if (mn.size() != 3 || mx.size() != 3 || nc.size() != 3)
        cfg::fail(CFG_ESETUP, "blockMesh: min/max/cells need 3 values each");
    const char* keys[6] = {"xmin", "xmax", "ymin", "ymax", "zmin", "zmax"};
    std::vector<std::string> names = {"xmin", "xmax", "ymin", "ymax", "zmin", "zmax"};
    std::vector<std::string> types = {"wall", "wall", "wall", "wall", "symmetry", "symmetry"};
    for (int s = 0; s < 6; ++s)
        if (b.has(keys[s]))
        {
            const cfg::Dict& sd = b.dict(keys[s]);
            names[s] = sd.wordOr("name", keys[s]);
            types[s] = sd.wordOr("type", "wall");
        }
    cs.mesh = cfg::blockMesh({mn[0], mn[1], mn[2]}, {mx[0], mx[1], mx[2]}, static_cast<int64_t>(nc[0]),
                             static_cast<int64_t>(nc[1]), static_cast<int64_t>(nc[2]), names, types);
    }
    const cfg::Mesh& M = cs.mesh;
    const size_t nP = M.patches.size();
    // the fields' defaults: every patch zeroGradient (volFields.cpp:46-50)
    cs.uType.assign(nP, CFG_BC_ZERO_GRADIENT);
    cs.pType.assign(nP, CFG_BC_ZERO_GRADIENT);
    cs.uVal.assign(nP, {0, 0, 0});
    cs.pVal.assign(nP, 0.0);
    // patches{} (simpleFoamApp.cpp:54-91)
    if (d.has("patches"))
    {
        const cfg::Dict& ps = d.dict("patches");
        for (const auto& name : ps.keys())
        {
            const cfg::Dict& pd = ps.dict(name);
            int patch = -1;
            for (size_t i = 0; i < nP; ++i)
                if (M.patches[i].name == name) patch = static_cast<int>(i);
            if (patch < 0) cfg::fail(CFG_ESETUP, "polyMesh: no patch named '" + name + "'");
            if (pd.has("U"))
            {
                const auto ul = pd.numbers("U");
                if (ul.size() != 3) cfg::fail(CFG_ESETUP, "patch U needs 3 values");
                cs.uType[patch] = bcFromName(pd.wordOr("UType", "fixedValue"));
                cs.uVal[patch] = {ul[0], ul[1], ul[2]};
            }
            else
            {
                const bool isWall = M.patches[patch].type == "wall";
                cs.uType[patch] = isWall ? CFG_BC_FIXED_VALUE : bcFromName(pd.wordOr("UType", "zeroGradient"));
            }
            if (pd.has("p"))
            {
                cs.pType[patch] = bcFromName(pd.wordOr("pType", "fixedValue"));
                cs.pVal[patch] = pd.number("p");
            }
            else
            {
                cs.pType[patch] = CFG_BC_ZERO_GRADIENT;
            }
        }
    }
    // initial{U} (caseInit.h:18-31)
    if (d.has("initial") && d.dict("initial").has("U"))
    {
        const auto u0 = d.dict("initial").numbers("U");
        cs.hasU0 = true;
        for (int i = 0; i < 3; ++i) cs.u0[i] = u0[i];
    }
    // schemes{} (fvMatrix.cpp:148-160)
    if (d.has("schemes"))
    {
        const cfg::Dict& s = d.dict("schemes");
        const std::string div = s.wordOr("div", "upwind");
        // unknown names fall back to upwind, as fvm::div's alpha selection does
        cs.schemes.div = div == "linear" ? CFG_DIV_LINEAR
                         : div == "blend" ? CFG_DIV_BLEND
                         : div == "linearUpwind" ? CFG_DIV_LINEAR_UPWIND
                                                 : CFG_DIV_UPWIND;
        cs.schemes.laplacian_corrected = s.wordOr("laplacian", "corrected") == "corrected";
        const std::string g = s.wordOr("grad", "corrected");
        cs.schemes.grad =
            g == "corrected" ? CFG_GRAD_CORRECTED : (g == "leastSquares" ? CFG_GRAD_LEAST_SQUARES : CFG_GRAD_LINEAR);
        cs.schemes.blend_coeff = s.numberOr("blendCoeff", 0.9);
    }
    // simple{} (SimpleSolver.h:13-64 defaults; simpleFoamApp.cpp:115-132,
    // linearTol / linearMaxIter read as multiCoupledApp.cpp:41-57 reads them)
    cfg_simple_controls& c = cs.ctl;
    c.max_iterations = 200;
    c.continuity_tol = 1e-6;
    c.linear_tol = 1e-7;
    c.linear_max_iter = 2000;
    c.non_orth_correctors = 2;
    c.relax_u = 0.7;
    c.relax_p = 0.3;
    c.p_ref_cell = -1;
    c.verbose = 1;
    c.nu = d.number("nu");
    if (d.has("simple"))
    {
        const cfg::Dict& s = d.dict("simple");
        c.max_iterations = static_cast<int32_t>(s.numberOr("maxIterations", c.max_iterations));
        c.continuity_tol = s.numberOr("continuityTol", c.continuity_tol);
        c.pcorr_tol = s.numberOr("pcorrTol", c.pcorr_tol);
        c.relax_u = s.numberOr("relaxU", c.relax_u);
        c.relax_p = s.numberOr("relaxP", c.relax_p);
        c.p_relax_start = s.numberOr("pRelaxStart", c.p_relax_start);
        c.non_orth_correctors = static_cast<int32_t>(s.numberOr("nonOrthCorrectors", c.non_orth_correctors));
        c.momentum_tol = s.numberOr("momentumTol", c.momentum_tol);
        c.linear_tol = s.numberOr("linearTol", c.linear_tol);
        c.linear_max_iter = static_cast<int32_t>(s.numberOr("linearMaxIter", c.linear_max_iter));
        if (s.has("force"))
        {
            const auto f = s.numbers("force");
            if (f.size() != 3) cfg::fail(CFG_ESETUP, "simple force needs 3 values");
            for (int i = 0; i < 3; ++i) c.body_force[i] = f[i];
        }
    }
    // turbulence{} (TurbulenceConfig::fromCase, turbulenceModel.cpp:41-56):
    // a missing block means laminar
    if (d.has("turbulence"))
    {
        const cfg::Dict& t = d.dict("turbulence");
        cs.turbModel = t.wordOr("model", cs.turbModel);
        cs.turbIntensity = t.numberOr("intensity", cs.turbIntensity);
        cs.turbLength = t.numberOr("lengthScale", cs.turbLength);
        cs.turbRelax = t.numberOr("relaxation", cs.turbRelax);
        cs.cDES = t.numberOr("C_DES", cs.cDES);
        cs.reOnset = t.numberOr("reOnset", cs.reOnset);
        cs.onsetWidth = t.numberOr("onsetWidth", cs.onsetWidth);
        cs.gammaRate = t.numberOr("gammaRate", cs.gammaRate);
        if (!(cs.turbIntensity >= 0)) cfg::fail(CFG_ESETUP, "turbulence: intensity must be non-negative");
        if (!(cs.turbRelax > 0 && cs.turbRelax <= 1)) cfg::fail(CFG_ESETUP, "turbulence: relaxation must be in (0, 1]");
        const std::string& m = cs.turbModel;
        if (m != "laminar" && m != "kEpsilon" && m != "kOmegaSST" && m != "des" && m != "gammaTransition")
            cfg::fail(CFG_ESETUP, "turbulence: unknown model '" + m +
                                      "' (laminar | kEpsilon | kOmegaSST | des | gammaTransition)");
    }
    // gpu{}: settings the reference does not have; defaults reproduce it
    if (d.has("gpu"))
    {
        const cfg::Dict& g = d.dict("gpu");
        const std::string pp = g.wordOr("pPreconditioner", "Jacobi");
        c.p_precond = pp == "DIC"    ? CFG_PRECOND_DIC
                      : pp == "AMG"  ? CFG_PRECOND_AMG
                      : pp == "IR32" ? CFG_PRECOND_IR32
                                     : CFG_PRECOND_JACOBI;
        const std::string up = g.wordOr("uPreconditioner", "Jacobi");
        if (up != "Jacobi" && up != "AMG")
            cfg::fail(CFG_ESETUP, "gpu: unknown uPreconditioner '" + up + "' (Jacobi | AMG)");
        c.u_precond = up == "AMG" ? CFG_PRECOND_AMG : CFG_PRECOND_JACOBI;
        c.p_ref_cell = static_cast<int64_t>(g.numberOr("pRefCell", -1));
        c.p_ref_value = g.numberOr("pRefValue", 0.0);
        c.verbose = static_cast<int32_t>(g.numberOr("verbose", 1));
    }
    return cs;
}

}  // namespace

extern "C" {

int cfg_case_inspect(const char* path, char* out, size_t size)
{
    return guard([&] {
        need(path && out && size, "cfg_case_inspect: null argument");
        const CaseSpec cs = parseCase(path);
        std::string s;
        char buf[256];
        auto add = [&](const char* fmt, auto... v) {
            std::snprintf(buf, sizeof buf, fmt, v...);
            s += buf;
        };
        add("cells %lld\nfaces %lld\ninternal %lld\n", static_cast<long long>(cs.mesh.nCells),
            static_cast<long long>(cs.mesh.nFaces()), static_cast<long long>(cs.mesh.nInternal()));
        for (size_t i = 0; i < cs.mesh.patches.size(); ++i)
            add("patch %s %s %lld %lld U %d %.17g %.17g %.17g p %d %.17g\n", cs.mesh.patches[i].name.c_str(),
                cs.mesh.patches[i].type.c_str(), static_cast<long long>(cs.mesh.patches[i].start),
                static_cast<long long>(cs.mesh.patches[i].size), cs.uType[i], cs.uVal[i][0], cs.uVal[i][1],
                cs.uVal[i][2], cs.pType[i], cs.pVal[i]);
        add("schemes %d %d %d %.17g\n", cs.schemes.div, cs.schemes.laplacian_corrected, cs.schemes.grad,
            cs.schemes.blend_coeff);
        const cfg_simple_controls& c = cs.ctl;
        add("simple %d %.17g %.17g %.17g %.17g %d %d %.17g %.17g %.17g\n", c.max_iterations, c.continuity_tol,
            c.pcorr_tol, c.momentum_tol, c.linear_tol, c.linear_max_iter, c.non_orth_correctors, c.relax_u, c.relax_p,
            c.p_relax_start);
        add("force %.17g %.17g %.17g\nnu %.17g\n", c.body_force[0], c.body_force[1], c.body_force[2], c.nu);
        add("gpu %d %lld %.17g %d\n", c.p_precond, static_cast<long long>(c.p_ref_cell), c.p_ref_value, c.u_precond);
        if (cs.hasU0) add("initialU %.17g %.17g %.17g\n", cs.u0[0], cs.u0[1], cs.u0[2]);
        add("turbulence %s %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", cs.turbModel.c_str(), cs.turbIntensity,
            cs.turbLength, cs.turbRelax, cs.cDES, cs.reOnset, cs.onsetWidth, cs.gammaRate);
        std::snprintf(out, size, "%s", s.c_str());
    });
}

int cfg_run_case_file(const char* path, int32_t device, cfg_simple_result* result, int64_t counts[5], double* U,
                      double* p, double* phi)
{
    return guard([&] {
        need(path && result, "cfg_run_case_file: null argument");
        const CaseSpec cs = parseCase(path);
        const cfg::Mesh& M = cs.mesh;
        cfg::Ctx ctx(M, device, nullptr);
        for (size_t i = 0; i < M.patches.size(); ++i)
        {
            const int pi = static_cast<int>(i);
            ctx.setPatchBC('U', pi, cs.uType[i], cs.uVal[i].data());
            ctx.setPatchBC('p', pi, cs.pType[i], &cs.pVal[i]);
        }
        // the initial flux (simpleFoamApp.cpp:93-95) and the seeded field
        ctx.initFlux(nullptr);
        if (cs.hasU0) ctx.initFlux(cs.u0);
        ctx.setSchemes(cs.schemes);
        // the RANS model, created after the initial flux (simpleFoamApp.cpp:93-102)
        if (cs.turbModel != "laminar")
        {
            ctx.turbulenceParams(cs.cDES, cs.reOnset, cs.onsetWidth, cs.gammaRate);
            ctx.turbulenceSetup(cs.turbModel.c_str(), cs.turbIntensity, cs.turbLength, cs.turbRelax, cs.ctl.nu);
        }
        ctx.iterate(cs.ctl, *result);
        if (counts)
        {
            counts[0] = static_cast<int64_t>(M.points.size());
            counts[1] = M.nCells;
            counts[2] = M.nFaces();
            counts[3] = M.nInternal();
            counts[4] = static_cast<int64_t>(M.patches.size());
        }
        ctx.download(U, p, phi);
    });
}

}  // extern "C"

// ---- detail blocks and batches ----

int cfg_detail_setup(cfg_ctx* ctx, const char* shape, double rho)
{
    return guard([&] {
        need(ctx && shape, "cfg_detail_setup: null argument");
        ctx->c->detailSetup(shape, rho);
    });
}

int cfg_detail_loss(cfg_ctx* ctx, double q, const cfg_simple_controls* controls, cfg_detail_measure* out)
{
    return guard([&] {
        need(ctx && controls && out, "cfg_detail_loss: null argument");
        ctx->c->detailLoss(q, *controls, *out);
        if (out->status != CFG_OK)
            cfg::fail(out->status, !std::isfinite(out->dp_pa)
                                       ? std::string("detailBlock: non-finite pressure drop")
                                       : "detailBlock: the detailed region reports a non-positive drop (" +
                                             std::to_string(out->dp_pa) + " Pa) at " + std::to_string(q) +
                                             " m3/s");
    });
}

int cfg_detail_turbulence(cfg_ctx* ctx, const char* model, double intensity, double lengthScale, double relaxation,
                          double nu)
{
    return guard([&] {
        need(ctx && model, "cfg_detail_turbulence: null argument");
        ctx->c->detailTurbulence(model, intensity, lengthScale, relaxation, nu);
    });
}

int cfg_batch_create(int32_t n, cfg_ctx* const* blocks, cfg_batch** out)
{
    return guard([&] {
        need(n > 0 && blocks && out, "cfg_batch_create: null argument or empty batch");
        auto b = std::make_unique<cfg_batch>();
        for (int32_t i = 0; i < n; ++i)
        {
            need(blocks[i] != nullptr, "cfg_batch_create: null block");
            for (int32_t j = 0; j < i; ++j) need(blocks[j] != blocks[i], "cfg_batch_create: a block appears twice");
            b->blocks.push_back(blocks[i]->c.get());
        }
        *out = b.release();
    });
}

void cfg_batch_destroy(cfg_batch* batch) { delete batch; }

int cfg_batch_set_schedule(cfg_batch* batch, int32_t workers, int32_t rowBlocks)
{
    return guard([&] {
        need(batch && workers >= 0 && rowBlocks >= -1, "cfg_batch_set_schedule: bad argument");
        batch->workers = workers;
        batch->rowBlocks = rowBlocks;
    });
}

int cfg_batch_loss(cfg_batch* batch, const double* q, const cfg_simple_controls* controls, cfg_detail_measure* out,
                   double* wallMs)
{
    return guard([&] {
        need(batch && q && controls && out, "cfg_batch_loss: null argument");
        cfg::batchPass(*batch, q, controls, out, wallMs);
    });
}

int cfg_batch_save(cfg_batch* batch)
{
    return guard([&] {
        need(batch, "cfg_batch_save: null argument");
        for (cfg::Ctx* c : batch->blocks) c->saveState();
    });
}

int cfg_batch_restore(cfg_batch* batch)
{
    return guard([&] {
        need(batch, "cfg_batch_restore: null argument");
        for (cfg::Ctx* c : batch->blocks) c->restoreState();
    });
}

int cfg_batch_autotune(cfg_batch* batch, const double* q, const cfg_simple_controls* controls, int32_t* workers,
                       int32_t* rowBlocks, double* times)
{
    return guard([&] {
        need(batch && q && controls && workers && rowBlocks, "cfg_batch_autotune: null argument");
        // {host workers, solver blocks per SM}; 0 workers: the pass as one
        // captured graph (Jacobi / DIC pressure, one outer iteration)
        static const int cand[][2] = {{1, 0}, {8, 1}, {16, 1}, {16, -1}, {32, -1}, {64, -1},
                                      {0, 1}, {0, 2}, {0, -1}};
        constexpr int nCand = sizeof(cand) / sizeof(cand[0]);
        bool graphable = true;
        for (size_t i = 0; i < batch->blocks.size(); ++i)
            graphable = graphable && controls[i].max_iterations == 1 && controls[i].p_precond != CFG_PRECOND_AMG &&
                        controls[i].u_precond == CFG_PRECOND_JACOBI &&
                        controls[i].p_precond != CFG_PRECOND_MPNN && controls[i].p_precond != CFG_PRECOND_IR32 &&
                        controls[i].p_precond != CFG_PRECOND_AMG_MPNN &&
                        batch->blocks[i]->turbulenceModelName() != "gammaTransition";
        std::vector<cfg_detail_measure> m(batch->blocks.size());
        double best = 0;
        int bi = 0;
        // every candidate runs the same pass from the same saved fields; the
        // chosen one then runs it for real
        for (cfg::Ctx* c : batch->blocks) c->saveState();
        for (int k = 0; k < nCand; ++k)
        {
            if (cand[k][0] == 0 && !graphable)
            {
                if (times) times[k] = -1.0;
                continue;
            }
            for (cfg::Ctx* c : batch->blocks) c->restoreState();
            batch->workers = cand[k][0];
            batch->rowBlocks = cand[k][1];
            double ms = 0;
            cfg::batchPass(*batch, q, controls, m.data(), &ms);
            // a schedule's first pass includes its first-time costs (graph
            // captures of the chunks, or of the whole pass): time a second
            // run of the same pass from the same fields
            for (cfg::Ctx* c : batch->blocks) c->restoreState();
            cfg::batchPass(*batch, q, controls, m.data(), &ms);
            if (times) times[k] = ms;
            if (k == 0 || ms < best)
            {
                best = ms;
                bi = k;
            }
        }
        for (cfg::Ctx* c : batch->blocks) c->restoreState();
        batch->workers = cand[bi][0];
        batch->rowBlocks = cand[bi][1];
        cfg::batchPass(*batch, q, controls, m.data(), nullptr);
        *workers = batch->workers;
        *rowBlocks = batch->rowBlocks;
    });
}

// ---- RANS turbulence ----

int cfg_turbulence_setup(cfg_ctx* ctx, const char* model, double intensity, double lengthScale, double relaxation,
                         double nu)
{
    return guard([&] {
        need(ctx && model, "cfg_turbulence_setup: null argument");
        ctx->c->refreshBcPublic();
        ctx->c->turbulenceSetup(model, intensity, lengthScale, relaxation, nu);
    });
}

int cfg_turbulence_params(cfg_ctx* ctx, double c_des, double re_onset, double onset_width, double gamma_rate)
{
    return guard([&] {
        need(ctx, "cfg_turbulence_params: null argument");
        ctx->c->turbulenceParams(c_des, re_onset, onset_width, gamma_rate);
    });
}

int cfg_turbulence_fields(cfg_ctx* ctx, double* k, double* eps, double* nut, double* nuEffFace)
{
    return guard([&] {
        need(ctx, "cfg_turbulence_fields: null argument");
        ctx->c->turbulenceFields(k, eps, nut, nuEffFace);
    });
}

// ---- learned pressure preconditioner ----

int cfg_mpnn_create(cfg_ctx* ctx, int32_t layers, uint64_t seed)
{
    return guard([&] {
        need(ctx, "cfg_mpnn_create: null argument");
        ctx->c->mpnnCreate(layers, seed);
    });
}

int cfg_mpnn_params(const cfg_ctx* ctx, int64_t* n)
{
    return guard([&] {
        need(ctx && n, "cfg_mpnn_params: null argument");
        *n = ctx->c->mpnnParams();
    });
}

int cfg_mpnn_weights(cfg_ctx* ctx, float* get, const float* set, int64_t n)
{
    return guard([&] {
        need(ctx, "cfg_mpnn_weights: null argument");
        ctx->c->mpnnWeights(get, set, n);
    });
}

int cfg_mpnn_loss_grad(cfg_ctx* ctx, const double* r, double* loss, float* grad)
{
    return guard([&] {
        need(ctx && r && loss, "cfg_mpnn_loss_grad: null argument");
        *loss = ctx->c->mpnnLossGradHost(r, grad);
    });
}

int cfg_mpnn_apply(cfg_ctx* ctx, const double* r, double* z)
{
    return guard([&] {
        need(ctx && r && z, "cfg_mpnn_apply: null argument");
        ctx->c->mpnnApplyHost(r, z);
    });
}

int cfg_mpnn_train(cfg_ctx* ctx, const double* samples, int32_t nSamples, int32_t epochs, float lr, double* losses)
{
    return guard([&] {
        need(ctx && samples, "cfg_mpnn_train: null argument");
        ctx->c->mpnnTrainHost(samples, nSamples, epochs, lr, losses);
    });
}

int cfg_mpnn_time(cfg_ctx* ctx, int32_t reps, double out[2])
{
    return guard([&] {
        need(ctx && out && reps > 0, "cfg_mpnn_time: bad argument");
        ctx->c->mpnnTime(reps, out);
    });
}

int cfg_mpnn_train_pairs(cfg_ctx* ctx, const double* samples, const double* targets, int32_t nSamples,
                         int32_t epochs, float lr, double* losses)
{
    return guard([&] {
        need(ctx && samples && targets, "cfg_mpnn_train_pairs: null argument");
        ctx->c->mpnnTrainHost(samples, nSamples, epochs, lr, losses, targets);
    });
}

int cfg_mpnn_loss_grad_pair(cfg_ctx* ctx, const double* r, const double* t, double* loss, float* grad)
{
    return guard([&] {
        need(ctx && r && t && loss, "cfg_mpnn_loss_grad_pair: null argument");
        *loss = ctx->c->mpnnLossGradHost(r, grad, t);
    });
}

int cfg_poisson_residual(cfg_ctx* ctx, const double* b, const double* x, double* r)
{
    return guard([&] {
        need(ctx && b && x && r, "cfg_poisson_residual: null argument");
        ctx->c->poissonResidual(b, x, r);
    });
}

// ---- PISO ----

int cfg_piso_step(cfg_ctx* ctx, const cfg_piso_controls* controls, cfg_piso_result* result)
{
    return guard([&] {
        need(ctx && controls && result, "cfg_piso_step: null argument");
        ctx->c->pisoStep(*controls, *result);
    });
}

// ---- VTK output ----

int cfg_write_vtu(cfg_ctx* ctx, const char* path, int32_t binary)
{
    return guard([&] {
        need(ctx && path, "cfg_write_vtu: null argument");
        cfg::Ctx& c = *ctx->c;
        const cfg::Mesh& M = c.mesh();
        const size_t nC = static_cast<size_t>(M.nCells);
        std::vector<cfg::VtuField> f;
        f.push_back({"p", 1, std::vector<double>(nC)});
        f.push_back({"U", 3, std::vector<double>(3 * nC)});
        c.download(f[1].data.data(), f[0].data.data(), nullptr);
        if (c.hasTurbulence())
        {
            // the dissipation variable under the model's own name
            const char* dn = c.turbulenceModelName() == "kOmegaSST" ? "omega" : "epsilon";
            f.insert(f.begin() + 1, {{"k", 1, std::vector<double>(nC)}, {dn, 1, std::vector<double>(nC)},
                                     {"nut", 1, std::vector<double>(nC)}});
            c.turbulenceFields(f[1].data.data(), f[2].data.data(), f[3].data.data(), nullptr);
        }
        cfg::writeVtu(M, path, f, binary != 0);
    });
}

int cfg_write_hdf5(cfg_ctx* ctx, const char* path)
{
    return guard([&] {
        need(ctx && path, "cfg_write_hdf5: null argument");
        cfg::Ctx& c = *ctx->c;
        const cfg::Mesh& M = c.mesh();
        const size_t nC = static_cast<size_t>(M.nCells);
        std::vector<double> p(nC), U(3 * nC), k, eps, nut;
        c.download(U.data(), p.data(), nullptr);
        std::vector<std::pair<std::string, const double*>> f{{"p", p.data()}};
        if (c.hasTurbulence())
        {
            k.resize(nC);
            eps.resize(nC);
            nut.resize(nC);
            c.turbulenceFields(k.data(), eps.data(), nut.data(), nullptr);
            f.push_back({"k", k.data()});
            f.push_back({c.turbulenceModelName() == "kOmegaSST" ? "omega" : "epsilon", eps.data()});
            f.push_back({"nut", nut.data()});
        }
        // U is cell-major (x y z per cell); the datasets are one component each
        std::vector<double> Uc(3 * nC);
        for (size_t i = 0; i < nC; ++i)
            for (size_t q = 0; q < 3; ++q) Uc[q * nC + i] = U[3 * i + q];
        f.push_back({"Ux", Uc.data()});
        f.push_back({"Uy", Uc.data() + nC});
        f.push_back({"Uz", Uc.data() + 2 * nC});
        cfg::writeHdf5(M, path, f);
    });
}

int cfg_mesh_write_hdf5(const cfg_mesh* mesh, const char* path, int32_t n_fields, const char* const* names,
                        const double* const* data)
{
    return guard([&] {
        need(mesh && path && n_fields >= 0 && (n_fields == 0 || (names && data)), "cfg_mesh_write_hdf5: null argument");
        std::vector<std::pair<std::string, const double*>> f;
        for (int32_t i = 0; i < n_fields; ++i)
        {
            need(names[i] && (data[i] || mesh->m.nCells == 0), "cfg_mesh_write_hdf5: null field");
            f.push_back({names[i], data[i]});
        }
        cfg::writeHdf5(mesh->m, path, f);
    });
}

int cfg_mesh_write_vtu(const cfg_mesh* mesh, const char* path, int32_t n_fields, const char* const* names,
                       const int32_t* n_comp, const double* const* data, int32_t binary)
{
    return guard([&] {
        need(mesh && path && (n_fields == 0 || (names && n_comp && data)), "cfg_mesh_write_vtu: null argument");
        const size_t nC = static_cast<size_t>(mesh->m.nCells);
        std::vector<cfg::VtuField> f;
        for (int32_t i = 0; i < n_fields; ++i)
        {
            need(n_comp[i] == 1 || n_comp[i] == 3, "cfg_mesh_write_vtu: fields have 1 or 3 components");
            f.push_back({names[i], n_comp[i], std::vector<double>(data[i], data[i] + nC * n_comp[i])});
        }
        cfg::writeVtu(mesh->m, path, f, binary != 0);
    });
}

int cfg_mpnn_collect(cfg_ctx* ctx, int32_t on, int32_t maxSamples, int32_t* n)
{
    return guard([&] {
        need(ctx, "cfg_mpnn_collect: null argument");
        ctx->c->mpnnCollect(on, maxSamples);
        if (n) *n = ctx->c->mpnnCollected();
    });
}

int cfg_mpnn_train_collected(cfg_ctx* ctx, int32_t epochs, float lr, double* losses)
{
    return guard([&] {
        need(ctx, "cfg_mpnn_train_collected: null argument");
        ctx->c->mpnnTrainCollected(epochs, lr, losses);
    });
}
