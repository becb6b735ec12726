// cf::gpu::solveIncompressibleSimple: the reference's fields and settings
// translated onto the chuanflow_b200 C ABI (see cf_simple_gpu.h).
#include "cf_simple_gpu.h"

#include <string>
#include <vector>

#include "cf_gpu_common.h"

namespace cf
{
namespace gpu
{
namespace
{

using detail::check;
using detail::toSchemes;

int bcType(const std::string& s)
{
    if (s == "fixedValue") return CFG_BC_FIXED_VALUE;
    if (s == "zeroGradient") return CFG_BC_ZERO_GRADIENT;
    if (s == "fixedGradient") return CFG_BC_FIXED_GRADIENT;
    if (s == "symmetry") return CFG_BC_SYMMETRY;
    if (s == "outlet") return CFG_BC_OUTLET;
    if (s == "wall") return CFG_BC_WALL;
    if (s == "empty") return CFG_BC_EMPTY;
    throw Error("chuanflow_b200: unknown patch bc type '" + s + "'");
}

}  // namespace

SimpleSession::SimpleSession(const polyMesh& mesh, const Options& opt) : mesh_(mesh), opt_(opt)
{
    const auto& pts = mesh.points();
    std::vector<double> xyz;
    xyz.reserve(3 * pts.size());
    for (const auto& v : pts)
    {
        xyz.push_back(v.x);
        xyz.push_back(v.y);
        xyz.push_back(v.z);
    }
    std::vector<std::int64_t> off{0}, verts;
    for (const auto& f : mesh.faces())
    {
        verts.insert(verts.end(), f.begin(), f.end());
        off.push_back(static_cast<std::int64_t>(verts.size()));
    }
    std::vector<std::string> names, types;
    std::vector<const char*> np, tp;
    std::vector<std::int64_t> start, size;
    for (const auto& pt : mesh.patches())
    {
        names.push_back(pt.name);
        types.push_back(pt.type);
        start.push_back(pt.start);
        size.push_back(pt.size);
    }
    for (std::size_t i = 0; i < names.size(); ++i)
    {
        np.push_back(names[i].c_str());
        tp.push_back(types[i].c_str());
    }
    check(cfg_mesh_create(xyz.data(), static_cast<std::int64_t>(pts.size()), off.data(), verts.data(),
                          mesh.nFaces(), mesh.owner().data(), mesh.neighbour().data(), mesh.nInternalFaces(),
                          static_cast<std::int32_t>(names.size()), np.data(), tp.data(), start.data(), size.data(),
                          &m_),
          "cfg_mesh_create");
    const int st = cfg_ctx_create(m_, opt.device, nullptr, &c_);
    if (st != CFG_OK)
    {
        cfg_mesh_destroy(m_);
        m_ = nullptr;
        check(st, "cfg_ctx_create");
    }
}

SimpleSession::~SimpleSession()
{
    if (c_) cfg_ctx_destroy(c_);
    if (m_) cfg_mesh_destroy(m_);
}

SimpleResult SimpleSession::solve(volVectorField& U, volScalarField& p, surfaceScalarField& phi, scalar nu,
                                  const Schemes& schemes, const SimpleControls& ctl)
{
    if (&U.mesh() != &mesh_ || &p.mesh() != &mesh_ || &phi.mesh() != &mesh_)
        throw Error("chuanflow_b200: fields belong to another mesh than the session's");
    if (ctl.cellForce) throw Error("chuanflow_b200: cell forces are not on the GPU SIMPLE path");
    // the time term's own checks (simpleSolver.cpp:75-97)
    if ((ctl.dt > 0 || ctl.uTimeOld) && schemes.ddt != "Euler")
        throw Error("SIMPLE: the momentum equation is asked to step in time while schemes ddt is '" + schemes.ddt +
                    "', not 'Euler'");

    // boundary conditions, patch by patch, then the per-face velocity values
    // (Fields.h:42, :90, :97): every face of a fixed-value U patch is sent
    // with the value the reference's field reports for it
    const label nPatch = static_cast<label>(mesh_.patches().size());
    std::vector<std::int64_t> faces;
    std::vector<double> fvals;
    for (label pi = 0; pi < nPatch; ++pi)
    {
        const Vector uv = U.patchValue(pi);
        const double u3[3] = {uv.x, uv.y, uv.z};
        const std::string ut = U.patchBcType(pi);
        check(cfg_set_patch_bc(c_, 'U', static_cast<std::int32_t>(pi), bcType(ut), u3), "cfg_set_patch_bc(U)");
        const double pv = p.patchValue(pi);
        check(cfg_set_patch_bc(c_, 'p', static_cast<std::int32_t>(pi), bcType(p.patchBcType(pi)), &pv),
              "cfg_set_patch_bc(p)");
        if (ut == "fixedValue")
        {
            const auto& pt = mesh_.patches()[static_cast<std::size_t>(pi)];
            for (label f = pt.start; f < pt.start + pt.size; ++f)
            {
                const Vector fv = U.faceValue(f);
                if (fv.x == uv.x && fv.y == uv.y && fv.z == uv.z) continue;
                faces.push_back(f);
                fvals.insert(fvals.end(), {fv.x, fv.y, fv.z});
            }
        }
    }
    check(cfg_clear_face_values_U(c_), "cfg_clear_face_values_U");
    if (!faces.empty())
        check(cfg_set_face_values_U(c_, static_cast<std::int64_t>(faces.size()), faces.data(), fvals.data()),
              "cfg_set_face_values_U");
    const cfg_schemes sc = toSchemes(schemes);
    check(cfg_set_schemes(c_, &sc), "cfg_set_schemes");

    const label nC = mesh_.nCells();
    std::vector<double> u(3 * static_cast<std::size_t>(nC));
    for (label c = 0; c < nC; ++c)
    {
        const Vector& v = U.internalField()[static_cast<std::size_t>(c)];
        u[3 * c] = v.x;
        u[3 * c + 1] = v.y;
        u[3 * c + 2] = v.z;
    }
    check(cfg_fields_upload(c_, u.data(), p.internalField().data(), phi.values().data()), "cfg_fields_upload");

    cfg_simple_controls cc = detail::toControls(ctl, nu);
    if (ctl.uTimeOld)
    {
        // the caller's velocity at the previous time level
        std::vector<double> uo(3 * static_cast<std::size_t>(nC));
        for (label c = 0; c < nC && static_cast<std::size_t>(c) < ctl.uTimeOld->size(); ++c)
        {
            const Vector& v = (*ctl.uTimeOld)[static_cast<std::size_t>(c)];
            uo[3 * c] = v.x;
            uo[3 * c + 1] = v.y;
            uo[3 * c + 2] = v.z;
        }
        if (ctl.uTimeOld->size() != static_cast<std::size_t>(nC))
            throw Error("SIMPLE: the old velocity carries " + std::to_string(ctl.uTimeOld->size()) +
                        " cells for a mesh of " + std::to_string(nC));
        check(cfg_fields_upload_old(c_, uo.data()), "cfg_fields_upload_old");
    }
    cc.p_precond = opt_.dicPressure ? CFG_PRECOND_DIC : CFG_PRECOND_JACOBI;
    cc.verbose = opt_.verbose ? 1 : 0;
    cc.p_ref_cell = opt_.pRefCell;
    cc.p_ref_value = opt_.pRefValue;
    cfg_simple_result r{};
    check(cfg_simple_iterate(c_, &cc, &r), "cfg_simple_iterate");

    check(cfg_fields_download(c_, u.data(), p.internalField().data(), phi.values().data()), "cfg_fields_download");
    for (label c = 0; c < nC; ++c)
        U.internalField()[static_cast<std::size_t>(c)] = Vector{u[3 * c], u[3 * c + 1], u[3 * c + 2]};

    SimpleResult out;
    out.iterations = r.iterations;
    out.finalContinuityError = r.final_continuity_error;
    out.finalMomentumResidual = r.final_momentum_residual;
    out.converged = r.converged != 0;
    return out;
}

SimpleResult solveIncompressibleSimple(polyMesh& mesh, volVectorField& U, volScalarField& p,
                                       surfaceScalarField& phi, scalar nu, const Schemes& schemes,
                                       const SimpleControls& ctl, IEddyViscosity* turb, IEnergyCoupling* energy,
                                       const Options& opt)
{
    if (turb || energy) throw Error("chuanflow_b200: turbulence and energy coupling are not on the GPU SIMPLE path");
    SimpleSession s(mesh, opt);
    return s.solve(U, p, phi, nu, schemes, ctl);
}

}  // namespace gpu
}  // namespace cf
