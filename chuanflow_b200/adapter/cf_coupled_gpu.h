// GPU partners for ChuanFlow's coupled 1D-3D network (src/coupling).
//
// cf::gpu::GpuDetailBlock is an ICoupledElement (CoupledNetwork.h:232-331)
// whose lossAt runs the detailed region on the device through the
// chuanflow_b200 C ABI: the DetailBlock pattern (coupledNetwork.cpp:462-877,
// 1080-1195) of one block kept on the GPU and warm-started pass after pass.
// It drops into solveCoupled1d3d (coupledNetwork.cpp:1401-) wherever a
// DetailBlock pointer went.
//
// cf::gpu::GpuDetailBlockBatch runs a whole coupling pass of many blocks at
// once (cfg_batch_loss) under the unchanged driver.  The driver asks its
// partners one after another, each at the rate the network solve of that
// pass gave its edge; the first request of a pass re-solves the same network
// (solveSteadyNetwork is a pure function of the network and its controls, so
// the rates are the driver's own, bit for bit), evaluates every block at its
// rate concurrently, and the later requests of the pass read their answers.
// A request at any other rate is evaluated on its own, as a single block.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "cf/coupling/CoupledNetwork.h"
#include "cf_simple_gpu.h"
#include "chuanflow_b200.h"

struct cfg_batch;

namespace cf
{
namespace gpu
{

/// A detailed region on the device.  Covers the DetailBlock configurations
/// of a Newtonian, steady, incompressible region: laminar or one of the RANS
/// models kEpsilon, kOmegaSST, des, gammaTransition; inlet profile "flat",
/// "parabolic" or "power1over7".  A case that declares
/// anything else (a rheology, phases, a compressible or thermal region, an
/// Euler ddt) is refused at construction with cf::Error.  The probe range of
/// DetailBlock only feeds diagnostics that solveCoupled1d3d does not read and
/// is not taken.
class GpuDetailBlock : public coupling::ICoupledElement
{
public:
    GpuDetailBlock(polyMesh mesh, scalar nu, scalar rho, const Schemes& schemes, const SimpleControls& ctl,
                   const TurbulenceConfig& turb, const std::string& inletShape = "flat", const Options& opt = {});
    ~GpuDetailBlock() override;
    GpuDetailBlock(const GpuDetailBlock&) = delete;
    GpuDetailBlock& operator=(const GpuDetailBlock&) = delete;

    /// DetailBlock::lossAt: the rate's boundary conditions, SIMPLE from the
    /// block's current fields, the measured drop.  Raises cf::Error where the
    /// reference raises (a non-positive rate, a non-finite or non-positive
    /// drop).
    scalar lossAt(scalar qMag) override;
    label lastSweeps() const override { return measure_.sweeps; }
    bool lastConverged() const override { return measure_.converged != 0; }

    /// The last lossAt's measurement (BlockMeasure's laminar part).
    const cfg_detail_measure& measure() const { return measure_; }
    const polyMesh& mesh() const { return mesh_; }
    cfg_ctx* context() const { return session_->context(); }
    const cfg_simple_controls& controls() const { return controls_; }

private:
    friend class GpuDetailBlockBatch;
    /// the answer of a batched pass, checked as lossAt checks its own
    scalar accept(const cfg_detail_measure& m);

    polyMesh mesh_;
    std::unique_ptr<SimpleSession> session_;
    cfg_simple_controls controls_{};
    cfg_detail_measure measure_{};
};

/// Batched coupling passes over blocks that stay owned by the caller.
/// `net`, `edges` and `netCtl` are the ones the caller hands
/// solveCoupled1d3d; `blocks[i]` partners `edges[i]`.  The network must stay
/// alive and unchanged between the driver's network solve and the end of its
/// per-edge loop, which solveCoupled1d3d guarantees.
class GpuDetailBlockBatch
{
public:
    GpuDetailBlockBatch(std::vector<GpuDetailBlock*> blocks, const OneDNetwork& net, std::vector<label> edges,
                        const SteadyControls& netCtl);
    ~GpuDetailBlockBatch();
    GpuDetailBlockBatch(const GpuDetailBlockBatch&) = delete;
    GpuDetailBlockBatch& operator=(const GpuDetailBlockBatch&) = delete;

    /// The partners to pass to solveCoupled1d3d, in edge order.
    std::vector<coupling::ICoupledElement*> elements();

    /// The schedule of cfg_batch_set_schedule: blocks in flight at once and
    /// the solver grid per block (0 = the context's own, -1 = by block size).
    /// The default, min(blocks, 16) in flight on their own grids, answers
    /// exactly as the blocks asked one by one; -1 trades that for speed on
    /// many small blocks.
    void setSchedule(int workers, int rowBlocksPerSm);

    /// Passes evaluated as a batch, and requests answered on their own.
    long batchedPasses() const { return batchedPasses_; }
    long singleRequests() const { return singleRequests_; }

private:
    class Element;
    scalar lossFor(std::size_t i, scalar q);

    std::vector<GpuDetailBlock*> blocks_;
    const OneDNetwork& net_;
    std::vector<label> edges_;
    SteadyControls netCtl_;
    cfg_batch* batch_ = nullptr;
    std::vector<std::unique_ptr<Element>> elements_;
    std::vector<double> q_;                  // the rates of the pass in hand
    std::vector<cfg_detail_measure> out_;    // its answers
    std::vector<char> pending_;              // answers not yet read
    long batchedPasses_ = 0;
    long singleRequests_ = 0;
};

}  // namespace gpu
}  // namespace cf
