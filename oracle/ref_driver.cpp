// Test-infrastructure driver around the reference implementation.
//
// This file is the checker's side of the parity tests: it is linked against
// the reference's own hot-path sources (compiled by oracle/Makefile into
// oracle/_ref/) and runs them on inputs written by the tests, dumping raw
// little-endian arrays (.f64 / .i64) that the tests compare with the CUDA
// path and with the C restatement in oracle/cfo.c.  Nothing in the product
// links or runs it.
//
// Modes (all take the case dictionary the reference app would read):
//   mesh   <case.dict> <out> [points.f64]             addressing + geometry
//   meshtime <case.dict>                              seconds to load the case's mesh, cells, faces
//   grad   <case.dict> <out> <points|-> <T.f64> <bvals.f64>
//                                                     fvc::grad, both overloads
//   simple <case.dict> <out> [points|-] [statedir]    solveIncompressibleSimple
//   rans   <case.dict> <out> [points|-]               the same with the case's RANS model
//   piso   <case.dict> <out> [points|-]               transient PISO steps (piso{} block), with the
//                                                     case's RANS model when it has a turbulence{}
//   vtk    <case.dict> <out.vtu> <points|-> <p.f64> <U.f64>   VtkWriter
//   eqns   <case.dict> <out> <points|-> <statedir>    UEqn / pEqn assembly probes
//   solve  <out> <n> <trip.i64> <tripv.f64> <diag.f64> <b.f64> <x0.f64> <cg|bicgstab> <tol> <maxIter>
//
// The SIMPLE set-up follows src/3d/apps/simpleFoamApp.cpp:54-132 (patch BCs,
// initial flux, schemes, controls) and additionally reads linearTol and
// linearMaxIter from simple{} the way src/coupling/apps/multiCoupledApp.cpp:41-57
// does.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "cf/common/Dictionary.h"
#include "cf/common/Matrix.h"
#include "cf/fvm/Fields.h"
#include "cf/fvm/FvMatrix.h"
#include "cf/fvm/MeshLoader.h"
#include "cf/fvm/PressureCorrection.h"
#include "cf/fvm/PisoSolver.h"
#include "cf/fvm/SimpleSolver.h"
#include "cf/fvm/VtkWriter.h"
#include "cf/turbulence/TurbulenceModel.h"

// Built as cf_adapter_driver, the simple mode runs the same case through the
// GPU drop-in (chuanflow_b200/adapter) instead of the reference's solver.
#ifdef CFG_ADAPTER
#include "cf_simple_gpu.h"
#define SIMPLE_SOLVE cf::gpu::solveIncompressibleSimple
#else
#define SIMPLE_SOLVE solveIncompressibleSimple
#endif

using namespace cf;

namespace
{

template <class T>
std::vector<T> readRaw(const std::string& path)
{
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open " + path);
    in.seekg(0, std::ios::end);
    const std::size_t bytes = static_cast<std::size_t>(in.tellg());
    in.seekg(0);
    std::vector<T> v(bytes / sizeof(T));
    in.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(bytes));
    return v;
}

template <class T>
void writeRaw(const std::string& path, const T* p, std::size_t n)
{
    std::ofstream out(path, std::ios::binary);
    out.write(reinterpret_cast<const char*>(p), static_cast<std::streamsize>(n * sizeof(T)));
}

void writeVec(const std::string& path, const Field<Vector>& v)
{
    std::vector<double> flat(v.size() * 3);
    for (std::size_t i = 0; i < v.size(); ++i)
    {
        flat[3 * i] = v[i].x;
        flat[3 * i + 1] = v[i].y;
        flat[3 * i + 2] = v[i].z;
    }
    writeRaw(path, flat.data(), flat.size());
}

void writeSca(const std::string& path, const Field<scalar>& v) { writeRaw(path, v.data(), v.size()); }

polyMesh loadMesh(const Dictionary& dict, const std::string& casePath, const std::string& pointsPath)
{
    polyMesh mesh = MeshLoader::fromCase(dict, casePath);
    if (!pointsPath.empty() && pointsPath != "-")
    {
        const auto flat = readRaw<double>(pointsPath);
        Field<Vector> pts(flat.size() / 3);
        for (std::size_t i = 0; i < pts.size(); ++i) pts[i] = {flat[3 * i], flat[3 * i + 1], flat[3 * i + 2]};
        mesh.movePoints(pts);
    }
    return mesh;
}

void dumpMesh(const polyMesh& mesh, const std::string& out)
{
    {
        std::ofstream c(out + "/counts.txt");
        c << mesh.nPoints() << " " << mesh.nCells() << " " << mesh.nFaces() << " "
          << mesh.nInternalFaces() << " " << mesh.nPatches() << "\n";
    }
    {
        std::ofstream pt(out + "/patches.txt");
        for (const auto& p : mesh.patches()) pt << p.name << " " << p.type << " " << p.start << " " << p.size << "\n";
    }
    writeVec(out + "/points.f64", mesh.points());
    std::vector<long long> off{0}, verts;
    for (const auto& f : mesh.faces())
    {
        for (label v : f) verts.push_back(v);
        off.push_back(static_cast<long long>(verts.size()));
    }
    writeRaw(out + "/face_offsets.i64", off.data(), off.size());
    writeRaw(out + "/face_verts.i64", verts.data(), verts.size());
    writeRaw(out + "/owner.i64", mesh.owner().data(), mesh.owner().size());
    writeRaw(out + "/neighbour.i64", mesh.neighbour().data(), mesh.neighbour().size());
    writeSca(out + "/V.f64", mesh.cellVolumes());
    writeVec(out + "/C.f64", mesh.cellCentres());
    writeVec(out + "/Cf.f64", mesh.faceCentres());
    writeVec(out + "/Sf.f64", mesh.faceSf());
    writeSca(out + "/magSf.f64", mesh.faceAreas());
    writeVec(out + "/d.f64", mesh.deltaCoeffVec());
    writeSca(out + "/invDist.f64", mesh.deltaCoeff());
    const Field<scalar> ow = makeInternalOwnerWeights(mesh);
    writeSca(out + "/ow.f64", ow);
    writeVec(out + "/skew.f64", makeFaceSkewVectors(mesh, ow));
    writeSca(out + "/gammaHarm.f64", harmonicFaceGamma(mesh, Field<scalar>(1, 1e-4)));
}

/// Patch set-up of src/3d/apps/simpleFoamApp.cpp:56-91.
void applyPatches(const Dictionary& caseDict, const polyMesh& mesh, volVectorField& U, volScalarField& p)
{
    if (!caseDict.has("patches")) return;
    const Dictionary& ps = caseDict.getDict("patches");
    for (const auto& name : ps.keys())
    {
        const Dictionary& pd = ps.getDict(name);
        const label patch = mesh.patchIdByName(name);
        if (pd.has("U"))
        {
            const auto ul = pd.getScalarList("U");
            U.setPatchValue(patch, pd.getWordOr("UType", "fixedValue"), Vector{ul[0], ul[1], ul[2]});
        }
        else
        {
            const bool isWall = mesh.patches()[static_cast<std::size_t>(patch)].type == "wall";
            U.setPatchValue(patch, isWall ? "fixedValue" : pd.getWordOr("UType", "zeroGradient"), Vector::zero());
        }
        if (pd.has("p")) p.setPatchValue(patch, pd.getWordOr("pType", "fixedValue"), pd.getScalar("p"));
        else p.setPatchValue(patch, "zeroGradient", 0.0);
    }
}

SimpleControls readControls(const Dictionary& caseDict)
{
    SimpleControls ctl;
    if (!caseDict.has("simple")) return ctl;
    const Dictionary& sd = caseDict.getDict("simple");
    ctl.maxIterations = static_cast<int>(sd.getScalarOr("maxIterations", ctl.maxIterations));
    ctl.continuityTol = sd.getScalarOr("continuityTol", ctl.continuityTol);
    ctl.pcorrTol = sd.getScalarOr("pcorrTol", ctl.pcorrTol);
    ctl.relaxU = sd.getScalarOr("relaxU", ctl.relaxU);
    ctl.relaxP = sd.getScalarOr("relaxP", ctl.relaxP);
    ctl.pRelaxStart = sd.getScalarOr("pRelaxStart", ctl.pRelaxStart);
    ctl.nonOrthCorrectors = static_cast<int>(sd.getScalarOr("nonOrthCorrectors", ctl.nonOrthCorrectors));
    ctl.momentumTol = sd.getScalarOr("momentumTol", ctl.momentumTol);
    ctl.linearTol = sd.getScalarOr("linearTol", ctl.linearTol);
    ctl.linearMaxIter = static_cast<int>(sd.getScalarOr("linearMaxIter", ctl.linearMaxIter));
    if (sd.has("force"))
    {
        const auto f = sd.getScalarList("force");
        ctl.bodyForce = Vector{f[0], f[1], f[2]};
    }
    return ctl;
}

void loadState(const std::string& dir, volVectorField& U, volScalarField& p, surfaceScalarField& phi)
{
    const auto u = readRaw<double>(dir + "/U.f64");
    const auto pp = readRaw<double>(dir + "/p.f64");
    const auto ph = readRaw<double>(dir + "/phi.f64");
    for (std::size_t i = 0; i < U.internalField().size(); ++i)
        U.internalField()[i] = {u[3 * i], u[3 * i + 1], u[3 * i + 2]};
    for (std::size_t i = 0; i < p.internalField().size(); ++i) p.internalField()[i] = pp[i];
    for (std::size_t i = 0; i < phi.values().size(); ++i) phi.values()[i] = ph[i];
}

/// the reference's mesh loading alone, timed (reader throughput)
int modeMeshTime(int argc, char** argv)
{
    const Dictionary dict = Dictionary::parseFile(argv[2]);
    const auto t0 = std::chrono::steady_clock::now();
    const polyMesh mesh = MeshLoader::fromCase(dict, argv[2]);
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cout << std::setprecision(6) << s << " " << mesh.nCells() << " " << mesh.nFaces() << "\n";
    return 0;
}

int modeMesh(int argc, char** argv)
{
    const Dictionary dict = Dictionary::parseFile(argv[2]);
    const polyMesh mesh = loadMesh(dict, argv[2], argc > 4 ? argv[4] : "");
    dumpMesh(mesh, argv[3]);
    return 0;
}

int modeGrad(int argc, char** argv)
{
    const Dictionary dict = Dictionary::parseFile(argv[2]);
    const polyMesh mesh = loadMesh(dict, argv[2], argv[4]);
    const std::string out = argv[3];
    const auto tvals = readRaw<double>(argv[5]);
    const auto bvals = readRaw<double>(argv[6]);
    Field<scalar> t(tvals.begin(), tvals.end());
    const label nInt = mesh.nInternalFaces();
    const Field<scalar> ow = makeInternalOwnerWeights(mesh);
    auto fn = [&](label f, const Field<scalar>& data) -> scalar
    {
        if (f < nInt)
        {
            const std::size_t u = static_cast<std::size_t>(f);
            return ow[u] * data[static_cast<std::size_t>(mesh.owner()[u])]
                 + (1.0 - ow[u]) * data[static_cast<std::size_t>(mesh.neighbour()[u])];
        }
        return bvals[static_cast<std::size_t>(f - nInt)];
    };
    volScalarField T(mesh, "T");
    for (label pi = 0; pi < mesh.nPatches(); ++pi) T.setPatchValue(pi, "fixedValue", 0.0);
    for (label f = nInt; f < mesh.nFaces(); ++f) T.setFaceValue(f, bvals[static_cast<std::size_t>(f - nInt)]);
    T.internalField() = t;
    for (const char* s : {"linear", "corrected", "leastSquares"})
    {
        writeVec(out + "/grad_fn_" + s + ".f64", fvc::grad(mesh, t, fn, s));
        writeVec(out + "/grad_vol_" + s + ".f64", fvc::grad(T, s));
    }
    return 0;
}

/// simple with the case's turbulence{} block: the model is created after the
/// boundary conditions and the initial flux (simpleFoamApp.cpp:93-102) and
/// advanced inside solveIncompressibleSimple; k, the dissipation, nut and
/// the wall layer are dumped next to U, p and phi.
int modeRans(int argc, char** argv)
{
    const Dictionary caseDict = Dictionary::parseFile(argv[2]);
    const std::string out = argv[3];
    polyMesh mesh = loadMesh(caseDict, argv[2], argc > 4 ? argv[4] : "");
    const scalar nu = caseDict.getScalar("nu");
    volVectorField U(mesh, "U");
    volScalarField p(mesh, "p");
    surfaceScalarField phi(mesh, "phi", 0.0);
    applyPatches(caseDict, mesh, U, p);
    phi.correctBoundaryFlux(U);
    const Schemes schemes = loadSchemes(caseDict);
    const SimpleControls ctl = readControls(caseDict);
    const TurbulenceConfig cfg = TurbulenceConfig::fromCase(caseDict);
    std::unique_ptr<RansModel> turb = RansModel::create(mesh, U, phi, nu, schemes, cfg);
    const auto t0 = std::chrono::steady_clock::now();
    const SimpleResult res = solveIncompressibleSimple(mesh, U, p, phi, nu, schemes, ctl, turb.get());
    const auto t1 = std::chrono::steady_clock::now();
    writeVec(out + "/U.f64", U.internalField());
    writeSca(out + "/p.f64", p.internalField());
    writeSca(out + "/phi.f64", phi.values());
    writeSca(out + "/k.f64", turb->k());
    writeSca(out + "/eps.f64", turb->dissipation());
    writeSca(out + "/nut.f64", turb->nut());
    writeSca(out + "/nuEffFace.f64", turb->nuEffFace());
    writeSca(out + "/wallUTau.f64", turb->wallUTau());
    writeSca(out + "/wallYPlus.f64", turb->wallYPlus());
    std::ofstream r(out + "/result.txt");
    r << std::setprecision(17) << res.iterations << " " << res.finalContinuityError << " "
      << res.finalMomentumResidual << " " << (res.converged ? 1 : 0) << " "
      << std::chrono::duration<double>(t1 - t0).count() << " " << mesh.nCells() << "\n";
    return 0;
}

/// transient PISO: the case's piso{} block (dt, correctors, continuityTol,
/// nonOrthCorrectors, linearTol, linearMaxIter, steps) from rest
int modePiso(int argc, char** argv)
{
    const Dictionary caseDict = Dictionary::parseFile(argv[2]);
    const std::string out = argv[3];
    polyMesh mesh = loadMesh(caseDict, argv[2], argc > 4 ? argv[4] : "");
    const scalar nu = caseDict.getScalar("nu");
    volVectorField U(mesh, "U");
    volScalarField p(mesh, "p");
    surfaceScalarField phi(mesh, "phi", 0.0);
    applyPatches(caseDict, mesh, U, p);
    phi.correctBoundaryFlux(U);
    const Schemes schemes = loadSchemes(caseDict);
    PisoControls ctl;
    const Dictionary& pd = caseDict.getDict("piso");
    ctl.dt = pd.getScalar("dt");
    ctl.correctors = static_cast<int>(pd.getScalarOr("correctors", ctl.correctors));
    ctl.continuityTol = pd.getScalarOr("continuityTol", ctl.continuityTol);
    ctl.nonOrthCorrectors = static_cast<int>(pd.getScalarOr("nonOrthCorrectors", ctl.nonOrthCorrectors));
    ctl.linearTol = pd.getScalarOr("linearTol", ctl.linearTol);
    ctl.linearMaxIter = static_cast<int>(pd.getScalarOr("linearMaxIter", ctl.linearMaxIter));
    const int steps = static_cast<int>(pd.getScalarOr("steps", 1));
    // a case with a turbulence{} block steps its RANS model with the flow
    std::unique_ptr<RansModel> turb;
    if (caseDict.has("turbulence"))
        turb = RansModel::create(mesh, U, phi, nu, schemes, TurbulenceConfig::fromCase(caseDict));
    std::ofstream r(out + "/result.txt");
    r << std::setprecision(17);
    for (int s = 0; s < steps; ++s)
    {
        const PisoStepResult res = solveTransientIncompressiblePiso(mesh, U, p, phi, nu, schemes, ctl, turb.get());
        r << res.correctorsUsed << " " << res.predictedContinuityError << " " << res.continuityError << " "
          << res.pressureCorrectionMax << " " << (res.converged ? 1 : 0) << "\n";
    }
    writeVec(out + "/U.f64", U.internalField());
    writeSca(out + "/p.f64", p.internalField());
    writeSca(out + "/phi.f64", phi.values());
    if (turb)
    {
        writeSca(out + "/k.f64", turb->k());
        writeSca(out + "/eps.f64", turb->dissipation());
        writeSca(out + "/nut.f64", turb->nut());
        writeSca(out + "/nuEffFace.f64", turb->nuEffFace());
    }
    return 0;
}

/// VtkWriter on the case's mesh with cell fields p (scalar) and U (vector)
/// read from raw FP64 files
int modeVtk(int argc, char** argv)
{
    const Dictionary caseDict = Dictionary::parseFile(argv[2]);
    polyMesh mesh = loadMesh(caseDict, argv[2], argv[4]);
    const auto pv = readRaw<double>(argv[5]);
    const auto uv = readRaw<double>(argv[6]);
    Field<scalar> p(pv.begin(), pv.end());
    Field<Vector> U(static_cast<std::size_t>(mesh.nCells()));
    for (std::size_t c = 0; c < U.size(); ++c) U[c] = Vector{uv[3 * c], uv[3 * c + 1], uv[3 * c + 2]};
    VtkWriter w(mesh);
    w.addCellScalar("p", p);
    w.addCellVector("U", U);
    w.write(argv[3]);
    return 0;
}

int modeSimple(int argc, char** argv)
{
    const Dictionary caseDict = Dictionary::parseFile(argv[2]);
    const std::string out = argv[3];
    polyMesh mesh = loadMesh(caseDict, argv[2], argc > 4 ? argv[4] : "");
    const scalar nu = caseDict.getScalar("nu");
    volVectorField U(mesh, "U");
    volScalarField p(mesh, "p");
    surfaceScalarField phi(mesh, "phi", 0.0);
    applyPatches(caseDict, mesh, U, p);
    phi.correctBoundaryFlux(U);
    if (caseDict.has("initial") && caseDict.getDict("initial").has("U"))
    {
        const auto v = caseDict.getDict("initial").getScalarList("U");
        for (Vector& u : U.internalField()) u = Vector{v[0], v[1], v[2]};
        updatePhiInternal(mesh, U, phi);
        phi.correctBoundaryFlux(U);
    }
    if (argc > 5) loadState(argv[5], U, p, phi);
    const Schemes schemes = loadSchemes(caseDict);
    const SimpleControls ctl = readControls(caseDict);
    // simple { dt ...; }: pseudo-time stepping through SimpleControls::dt and
    // uTimeOld -- each of the maxIterations outer iterations is its own call
    // with one sweep, the velocity at the call's start as the old level
    const double pseudoDt = caseDict.getDict("simple").getScalarOr("dt", 0.0);

    const auto t0 = std::chrono::steady_clock::now();
    SimpleResult res;
    if (pseudoDt > 0)
    {
        Schemes eul = schemes;
        eul.ddt = "Euler";
        SimpleControls one = ctl;
        one.maxIterations = 1;
        one.dt = pseudoDt;
        int done = 0;
        for (int k = 0; k < ctl.maxIterations; ++k)
        {
            const Field<Vector> uOld = U.internalField();
            one.uTimeOld = &uOld;
            res = SIMPLE_SOLVE(mesh, U, p, phi, nu, eul, one);
            ++done;
            if (!std::isfinite(res.finalContinuityError)) break;
        }
        res.iterations = done;
    }
    else
    {
        res = SIMPLE_SOLVE(mesh, U, p, phi, nu, schemes, ctl);
    }
    const auto t1 = std::chrono::steady_clock::now();
    const double secs = std::chrono::duration<double>(t1 - t0).count();

    writeVec(out + "/U.f64", U.internalField());
    writeSca(out + "/p.f64", p.internalField());
    writeSca(out + "/phi.f64", phi.values());
    std::ofstream r(out + "/result.txt");
    r << std::setprecision(17) << res.iterations << " " << res.finalContinuityError << " "
      << res.finalMomentumResidual << " " << (res.converged ? 1 : 0) << " " << secs << " "
      << mesh.nCells() << "\n";
    return 0;
}

/// Assembly probes.  The momentum and pressure equations are built exactly as
/// src/3d/src/solvers/simpleSolver.cpp:67-115 and :260-274 build them, then
/// solved with maxIter 0 and one pass, so the CSR matrices exist and the rhs
/// holds the base source plus the corrector evaluated on the zero start.  The
/// explicit operator h = rhs - (A x - diag x) is then read at x = 0 and at a
/// probe vector, which pins the assembled rhs and the off-diagonal product.
int modeEqns(int argc, char** argv)
{
    const Dictionary caseDict = Dictionary::parseFile(argv[2]);
    const std::string out = argv[3];
    polyMesh mesh = loadMesh(caseDict, argv[2], argv[4]);
    const std::string state = argv[5];
    const scalar nu = caseDict.getScalar("nu");
    volVectorField U(mesh, "U");
    volScalarField p(mesh, "p");
    surfaceScalarField phi(mesh, "phi", 0.0);
    applyPatches(caseDict, mesh, U, p);
    loadState(state, U, p, phi);
    const Schemes schemes = loadSchemes(caseDict);
    const SimpleControls ctl = readControls(caseDict);
    const auto probe = readRaw<double>(state + "/xprobe.f64");
    Field<scalar> xprobe(probe.begin(), probe.end());
    Field<scalar> zero(xprobe.size(), 0.0);
    const label nC = mesh.nCells();
    const auto& vol = mesh.cellVolumes();

    const Field<Vector> gradPn = fvc::grad(p, schemes.grad);
    writeVec(out + "/gradPn.f64", gradPn);
    fvMatrix UEqn(mesh, viewOf(U), "UEqn");
    UEqn.schemes() = schemes;
    UEqn.schemes().relaxation = 1.0;
    fvm::div(UEqn, phi.values(), schemes.div);
    fvm::laplacian(UEqn, nu, schemes.laplacian, -1);
    for (label c = 0; c < nC; ++c)
    {
        const std::size_t u = static_cast<std::size_t>(c);
        const Vector rhs = vol[u] * (ctl.bodyForce + Vector::zero() - gradPn[u]);
        for (int comp = 0; comp < 3; ++comp) UEqn.addRhs(c, comp, rhs[comp]);
    }
    UEqn.solve(fvMatrix::Controls{ctl.linearTol, 0, 0});
    for (int comp = 0; comp < 3; ++comp)
    {
        Field<scalar> h;
        writeSca(out + "/U_diag" + std::to_string(comp) + ".f64", UEqn.aDiag(comp));
        UEqn.explicitOperator(zero, comp, h);
        writeSca(out + "/U_h0_" + std::to_string(comp) + ".f64", h);
        UEqn.explicitOperator(xprobe, comp, h);
        writeSca(out + "/U_h1_" + std::to_string(comp) + ".f64", h);
    }

    Field<scalar> rAUr(static_cast<std::size_t>(nC));
    const Field<scalar>& d = UEqn.aDiag(0);
    for (label c = 0; c < nC; ++c)
        rAUr[static_cast<std::size_t>(c)] = vol[static_cast<std::size_t>(c)] / std::max(d[static_cast<std::size_t>(c)], 1e-300);
    const Field<scalar> rAUf = interpolateToFaces(mesh, rAUr);
    writeSca(out + "/rAUf.f64", rAUf);
    const Field<scalar> divPhi = fvc::divPhi(mesh, phi.values());
    writeSca(out + "/divPhi.f64", divPhi);
    const scalar contErr = continuityError(mesh, phi);
    writeRaw(out + "/contErr.f64", &contErr, 1);
    volScalarField pFull(mesh, "pFull");
    for (label patch = 0; patch < mesh.nPatches(); ++patch)
        pFull.setPatchValue(patch, p.patchBcType(patch), p.patchValue(patch));
    fvMatrix pEqn(mesh, viewOf(pFull), "pEqn");
    pEqn.schemes() = schemes;
    pEqn.schemes().relaxation = 1.0;
    fvm::laplacianFace(pEqn, rAUf, schemes.laplacian, -1);
    for (label c = 0; c < nC; ++c) pEqn.addRhs(c, 0, -divPhi[static_cast<std::size_t>(c)]);
    pEqn.solve(fvMatrix::Controls{ctl.linearTol, 0, 0});
    {
        Field<scalar> h;
        writeSca(out + "/p_diag.f64", pEqn.aDiag(0));
        pEqn.explicitOperator(zero, 0, h);
        writeSca(out + "/p_h0.f64", h);
        pEqn.explicitOperator(xprobe, 0, h);
        writeSca(out + "/p_h1.f64", h);
    }
    // flux correction with the probe as the solved pressure
    for (label c = 0; c < nC; ++c) pFull.internalField()[static_cast<std::size_t>(c)] = xprobe[static_cast<std::size_t>(c)];
    const Field<Vector> gradPFull = fvc::grad(pFull, schemes.grad);
    writeVec(out + "/gradPFull.f64", gradPFull);
    surfaceScalarField phiC = phi;
    correctFluxes(mesh, pFull, gradPFull, rAUf, schemes, phiC);
    writeSca(out + "/phiCorrected.f64", phiC.values());
    return 0;
}

int modeSolve(int argc, char** argv)
{
    const std::string out = argv[2];
    const label n = std::atoll(argv[3]);
    const auto trip = readRaw<long long>(argv[4]);
    const auto tripv = readRaw<double>(argv[5]);
    const auto diag = readRaw<double>(argv[6]);
    const auto b = readRaw<double>(argv[7]);
    const auto x0 = readRaw<double>(argv[8]);
    const std::string method = argv[9];
    const double tol = std::atof(argv[10]);
    const int maxIter = std::atoi(argv[11]);
    SparseMatrix::Builder builder(n);
    for (std::size_t k = 0; k < tripv.size(); ++k) builder.add(trip[2 * k], trip[2 * k + 1], tripv[k]);
    const SparseMatrix A = builder.finishWithDiagonal(diag);
    Field<double> bb(b.begin(), b.end()), x(x0.begin(), x0.end());
    const auto t0 = std::chrono::steady_clock::now();
    const SolverReport rep = method == "cg" ? solveCG(A, bb, x, tol, maxIter) : solveBiCGStab(A, bb, x, tol, maxIter);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    writeSca(out + "/x.f64", x);
    std::ofstream r(out + "/report.txt");
    r << std::setprecision(17) << rep.iterations << " " << rep.initialResidual << " " << rep.finalResidual << " "
      << (rep.converged ? 1 : 0) << " " << secs << "\n";
    return 0;
}

} // namespace

int main(int argc, char** argv)
{
    if (argc < 3)
    {
        std::cerr << "usage: cf_ref_driver <mesh|grad|simple|eqns|solve> ...\n";
        return 2;
    }
    try
    {
        const std::string mode = argv[1];
        if (mode == "mesh" && argc >= 4) return modeMesh(argc, argv);
        if (mode == "meshtime" && argc >= 3) return modeMeshTime(argc, argv);
        if (mode == "grad" && argc >= 7) return modeGrad(argc, argv);
        if (mode == "simple" && argc >= 4) return modeSimple(argc, argv);
        if (mode == "rans" && argc >= 4) return modeRans(argc, argv);
        if (mode == "piso" && argc >= 4) return modePiso(argc, argv);
        if (mode == "vtk" && argc >= 7) return modeVtk(argc, argv);
        if (mode == "eqns" && argc >= 6) return modeEqns(argc, argv);
        if (mode == "solve" && argc >= 12) return modeSolve(argc, argv);
        std::cerr << "cf_ref_driver: bad arguments for mode " << mode << "\n";
        return 2;
    }
    catch (const std::exception& e)
    {
        std::cerr << "cf_ref_driver: " << e.what() << "\n";
        return 1;
    }
}
