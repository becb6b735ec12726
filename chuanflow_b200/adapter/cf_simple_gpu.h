// Drop-in C++ entry point for ChuanFlow's src/3d SIMPLE path, backed by the
// chuanflow_b200 C ABI.  Compiled inside the reference tree (it includes the
// reference's own headers) and linked with libchuanflow_b200.so, it lets a
// caller of cf::solveIncompressibleSimple (simpleFoamApp.cpp:140,
// coupledNetwork.cpp:1141, ns_bind.cpp:294, dpmApp.cpp) switch to the GPU by
// changing the namespace of one call.
#pragma once

#include <cstdint>
#include <memory>

#include "cf/fvm/SimpleSolver.h"

struct cfg_mesh;
struct cfg_ctx;

namespace cf
{
namespace gpu
{

/// Settings with no counterpart in SimpleControls; the defaults reproduce the
/// reference (Jacobi-PCG pressure, no reference cell).
struct Options
{
    int device = 0;
    bool dicPressure = false;   // multicolour DIC instead of Jacobi for the pressure PCG
    std::int64_t pRefCell = -1; // OpenFOAM-style pressure reference cell, -1 = none
    scalar pRefValue = 0;
    bool verbose = false;       // the reference's per-iteration log line
};

/// A mesh uploaded once to a device, reused by every solve on it (the
/// pattern of DetailBlock::lossAt, which re-solves one block many times).
/// The polyMesh must outlive the session and keep its topology and points.
class SimpleSession
{
public:
    SimpleSession(const polyMesh& mesh, const Options& opt = {});
    ~SimpleSession();
    SimpleSession(const SimpleSession&) = delete;
    SimpleSession& operator=(const SimpleSession&) = delete;

    /// solveIncompressibleSimple on this session's device: U, p and phi are
    /// read, iterated and written back in place, as the reference does.
    SimpleResult solve(volVectorField& U, volScalarField& p, surfaceScalarField& phi, scalar nu,
                       const Schemes& schemes, const SimpleControls& ctl);

    /// The session's C ABI context (owned by the session), for the calls
    /// this class does not wrap: detail blocks, batches, turbulence.
    cfg_ctx* context() const { return c_; }

private:
    const polyMesh& mesh_;
    Options opt_;
    cfg_mesh* m_ = nullptr;
    cfg_ctx* c_ = nullptr;
};

/// The reference's signature (SimpleSolver.h:119-127).  Turbulence and energy
/// coupling are not on this path: a non-null `turb` or `energy`, a cell force
/// or a time step is rejected with cf::Error, as is any input the reference
/// itself rejects (the C ABI's error message is carried through).
SimpleResult solveIncompressibleSimple(polyMesh& mesh, volVectorField& U, volScalarField& p,
                                       surfaceScalarField& phi, scalar nu, const Schemes& schemes,
                                       const SimpleControls& ctl, IEddyViscosity* turb = nullptr,
                                       IEnergyCoupling* energy = nullptr, const Options& opt = {});

}  // namespace gpu
}  // namespace cf
