// cf::gpu::GpuDetailBlock and GpuDetailBlockBatch (see cf_coupled_gpu.h).
#include "cf_coupled_gpu.h"

#include <algorithm>
#include <cmath>
#include <string>
#include <utility>

#include "cf_gpu_common.h"

namespace cf
{
namespace gpu
{

using detail::check;

GpuDetailBlock::GpuDetailBlock(polyMesh mesh, scalar nu, scalar rho, const Schemes& schemes,
                               const SimpleControls& ctl, const TurbulenceConfig& turb,
                               const std::string& inletShape, const Options& opt)
    : mesh_(std::move(mesh))
{
    // the checks of the DetailBlock constructor this block's scope reaches
    // (coupledNetwork.cpp:490-492, 514-517)
    if (!(nu > 0) || !(rho > 0)) throw Error("detailBlock: nu and rho must be positive");
    turb.validate();
    if (schemes.ddt != "steady")
        throw Error("chuanflow_b200: a detail block that carries its own du/dt (ddt " + schemes.ddt +
                    ") is not on the GPU path");
    if (ctl.cellForce || ctl.dt != 0 || ctl.uTimeOld)
        throw Error("chuanflow_b200: cell forces and time steps are not on the GPU SIMPLE path");
    session_ = std::make_unique<SimpleSession>(mesh_, opt);
    cfg_ctx* c = session_->context();
    const cfg_schemes sc = detail::toSchemes(schemes);
    check(cfg_set_schemes(c, &sc), "cfg_set_schemes");
    check(cfg_detail_setup(c, inletShape.c_str(), rho), "cfg_detail_setup");
    check(cfg_turbulence_params(c, turb.cDES, turb.reOnset, turb.onsetWidth, turb.gammaRate), "cfg_turbulence_params");
    if (turb.model != "laminar")
        check(cfg_detail_turbulence(c, turb.model.c_str(), turb.intensity, turb.lengthScale, turb.relaxation, nu),
              "cfg_detail_turbulence");
    controls_ = detail::toControls(ctl, nu);
    controls_.p_precond = opt.dicPressure ? CFG_PRECOND_DIC : CFG_PRECOND_JACOBI;
    controls_.verbose = opt.verbose ? 1 : 0;
    controls_.p_ref_cell = opt.pRefCell;
    controls_.p_ref_value = opt.pRefValue;
}

GpuDetailBlock::~GpuDetailBlock() = default;

scalar GpuDetailBlock::accept(const cfg_detail_measure& m)
{
    measure_ = m;
    // lossAt's checks of the measured drop (coupledNetwork.cpp:1146-1151)
    if (!std::isfinite(m.dp_pa)) throw Error("detailBlock: non-finite pressure drop");
    if (m.dp_pa <= 0)
        throw Error("detailBlock: the detailed region reports a non-positive drop (" + std::to_string(m.dp_pa) +
                    " Pa) at " + std::to_string(m.imposed_q) + " m3/s");
    return m.dp_pa;
}

scalar GpuDetailBlock::lossAt(scalar qMag)
{
    if (!(qMag > 0))
        throw Error("detailBlock: asked for the drop of a detailed region at a non-positive rate (" +
                    std::to_string(qMag) + " m3/s)");
    cfg_detail_measure m{};
    const int st = cfg_detail_loss(session_->context(), qMag, &controls_, &m);
    if (st != CFG_OK && st != CFG_ENUMERIC) check(st, "cfg_detail_loss");
    return accept(m);
}

/// One partner of the batch: block i, answered from the pass in hand.
class GpuDetailBlockBatch::Element : public coupling::ICoupledElement
{
public:
    Element(GpuDetailBlockBatch& b, std::size_t i) : b_(b), i_(i) {}
    scalar lossAt(scalar qMag) override { return b_.lossFor(i_, qMag); }
    label lastSweeps() const override { return b_.blocks_[i_]->lastSweeps(); }
    bool lastConverged() const override { return b_.blocks_[i_]->lastConverged(); }

private:
    GpuDetailBlockBatch& b_;
    std::size_t i_;
};

GpuDetailBlockBatch::GpuDetailBlockBatch(std::vector<GpuDetailBlock*> blocks, const OneDNetwork& net,
                                         std::vector<label> edges, const SteadyControls& netCtl)
    : blocks_(std::move(blocks)), net_(net), edges_(std::move(edges)), netCtl_(netCtl)
{
    if (blocks_.empty() || blocks_.size() != edges_.size())
        throw Error("chuanflow_b200: a batch needs one block per coupled edge");
    std::vector<cfg_ctx*> ctx;
    for (GpuDetailBlock* b : blocks_)
    {
        if (!b) throw Error("chuanflow_b200: a batch block is null");
        ctx.push_back(b->context());
    }
    check(cfg_batch_create(static_cast<int32_t>(ctx.size()), ctx.data(), &batch_), "cfg_batch_create");
    // up to 16 blocks in flight, each on its own solver grid: the answers are
    // those of the blocks asked one by one, bit for bit
    setSchedule(static_cast<int>(std::min<std::size_t>(blocks_.size(), 16)), 0);
    for (std::size_t i = 0; i < blocks_.size(); ++i) elements_.push_back(std::make_unique<Element>(*this, i));
    q_.assign(blocks_.size(), 0.0);
    out_.assign(blocks_.size(), cfg_detail_measure{});
    pending_.assign(blocks_.size(), 0);
}

GpuDetailBlockBatch::~GpuDetailBlockBatch()
{
    if (batch_) cfg_batch_destroy(batch_);
}

std::vector<coupling::ICoupledElement*> GpuDetailBlockBatch::elements()
{
    std::vector<coupling::ICoupledElement*> v;
    for (auto& e : elements_) v.push_back(e.get());
    return v;
}

void GpuDetailBlockBatch::setSchedule(int workers, int rowBlocksPerSm)
{
    check(cfg_batch_set_schedule(batch_, workers, rowBlocksPerSm), "cfg_batch_set_schedule");
}

scalar GpuDetailBlockBatch::lossFor(std::size_t i, scalar q)
{
    if (!(pending_[i] && q_[i] == q))
    {
        // a new pass: the rates the driver's own network solve gave every
        // coupled edge (the reference reads |flowRate| of each, :1462-1467)
        const SteadyNetworkResult res = solveSteadyNetwork(net_, netCtl_);
        std::vector<double> qs(edges_.size(), 0.0);
        bool usable = res.converged;
        for (std::size_t j = 0; j < edges_.size() && usable; ++j)
        {
            const label e = edges_[j];
            usable = e >= 0 && static_cast<std::size_t>(e) < res.pipeFlows.size();
            if (usable) qs[j] = std::abs(res.pipeFlows[static_cast<std::size_t>(e)].flowRate);
            usable = usable && qs[j] > 0;
        }
        if (!usable || qs[i] != q)
        {
            // not a pass of this network: this block alone
            ++singleRequests_;
            pending_[i] = 0;
            return blocks_[i]->lossAt(q);
        }
        std::vector<cfg_simple_controls> ctl;
        for (GpuDetailBlock* b : blocks_) ctl.push_back(b->controls());
        const int st = cfg_batch_loss(batch_, qs.data(), ctl.data(), out_.data(), nullptr);
        check(st, "cfg_batch_loss");
        q_ = qs;
        pending_.assign(blocks_.size(), 1);
        ++batchedPasses_;
    }
    pending_[i] = 0;
    return blocks_[i]->accept(out_[i]);
}

}  // namespace gpu
}  // namespace cf
