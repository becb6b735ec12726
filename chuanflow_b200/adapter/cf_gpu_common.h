// Helpers shared by the C++ drop-ins (cf_simple_gpu.cpp, cf_coupled_gpu.cpp):
// the reference's settings translated onto the chuanflow_b200 C ABI, and its
// error codes turned into the reference's exception type.
#pragma once

#include <string>

#include "cf/common/Error.h"
#include "cf/fvm/FvMatrix.h"
#include "cf/fvm/SimpleSolver.h"
#include "chuanflow_b200.h"

namespace cf
{
namespace gpu
{
namespace detail
{

/// A C ABI status other than CFG_OK as cf::Error, with the library's message.
inline void check(int status, const char* what)
{
    if (status == CFG_OK) return;
    char buf[1024];
    cfg_last_error(buf, sizeof buf);
    throw Error(std::string("chuanflow_b200 ") + what + ": " + buf);
}

/// Scheme names onto the ABI's enums.  Names the reference does not know
/// select its defaults, as its own string tests do (divScheme.cpp:18,
/// laplacianScheme.cpp:71, gradScheme.cpp:251-275); "linearUpwind" is this
/// library's extension.
inline cfg_schemes toSchemes(const Schemes& s)
{
    cfg_schemes out{};
    out.div = s.div == "linear" ? CFG_DIV_LINEAR
              : s.div == "blend" ? CFG_DIV_BLEND
              : s.div == "linearUpwind" ? CFG_DIV_LINEAR_UPWIND
                                        : CFG_DIV_UPWIND;
    out.laplacian_corrected = s.laplacian == "corrected" ? 1 : 0;
    out.grad = s.grad == "leastSquares" ? CFG_GRAD_LEAST_SQUARES
               : s.grad == "corrected" ? CFG_GRAD_CORRECTED
                                       : CFG_GRAD_LINEAR;
    out.blend_coeff = s.blendCoeff;
    return out;
}

/// SimpleControls (SimpleSolver.h:13-64) and nu onto the ABI's controls;
/// the GPU-only settings keep their reference-reproducing defaults unless
/// the caller sets them afterwards.
inline cfg_simple_controls toControls(const SimpleControls& ctl, scalar nu)
{
    cfg_simple_controls cc{};
    cc.max_iterations = ctl.maxIterations;
    cc.continuity_tol = ctl.continuityTol;
    cc.pcorr_tol = ctl.pcorrTol;
    cc.momentum_tol = ctl.momentumTol;
    cc.linear_tol = ctl.linearTol;
    cc.linear_max_iter = ctl.linearMaxIter;
    cc.non_orth_correctors = ctl.nonOrthCorrectors;
    cc.relax_u = ctl.relaxU;
    cc.relax_p = ctl.relaxP;
    cc.p_relax_start = ctl.pRelaxStart;
    cc.body_force[0] = ctl.bodyForce.x;
    cc.body_force[1] = ctl.bodyForce.y;
    cc.body_force[2] = ctl.bodyForce.z;
    cc.nu = nu;
    cc.p_precond = CFG_PRECOND_JACOBI;
    cc.verbose = 0;
    cc.p_ref_cell = -1;
    cc.p_ref_value = 0.0;
    cc.dt = ctl.dt;
    cc.u_time_old = ctl.uTimeOld ? 2 : 0;
    return cc;
}

}  // namespace detail
}  // namespace gpu
}  // namespace cf
