// Test-infrastructure driver for the coupled 1D-3D network.
//
// It builds a small 1D network whose middle is a set of parallel coupled
// edges, each partnered by a detailed 3D block, and runs the reference's
// steady interface iteration solveCoupled1d3d (coupledNetwork.cpp:1401-)
// on it.  Built twice by oracle/Makefile:
//
//   _ref/cf_coupled_driver <case.dict> <out>
//       the partners are the reference's own DetailBlock (CPU);
//   _ref/cf_coupled_gpu_driver <case.dict> <out> <single|batch>
//       the partners are chuanflow_b200/adapter's GpuDetailBlock, asked one
//       by one (single) or through GpuDetailBlockBatch (batch).
//
// Everything else (the network, the driver, its stop rule) is the
// reference's code, so the two runs differ only in who answers lossAt.
// Output: <out>/history.txt, one line per pass and edge
//   "pass edge q dpPa resistance sweeps blockConverged"
// then "result iterations converged residual", all at 17 digits; in batch
// mode <out>/batch.txt holds "batchedPasses singleRequests".
//
// The case dictionary:
//   network  { qIn; pOut; rho; mu; rIn; rOut; }      rate qIn into Src, pressure pOut at Snk:
//                                                     Src -In- J1 -{coupled}- J2 -Out- Snk
//   coupling { maxOuterIterations; relax; tolerance; accelerate; networkTol; }
//   schemes  { ... }   simple { ... }                 as the reference's case files
//   blocks   { <edge name> { block { ... }; nu; rho; shape; resistance;
//                            turbulence { ... } } ... }
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "cf/common/Dictionary.h"
#include "cf/coupling/CoupledNetwork.h"
#include "cf/fvm/MeshLoader.h"
#include "cf/turbulence/TurbulenceModel.h"

#ifdef CFG_ADAPTER
#include "cf_coupled_gpu.h"
#endif

using namespace cf;

namespace
{

SimpleControls controlsOf(const Dictionary& caseDict)
{
    SimpleControls c;
    if (!caseDict.has("simple")) return c;
    const Dictionary& s = caseDict.getDict("simple");
    c.maxIterations = static_cast<int>(s.getScalarOr("maxIterations", c.maxIterations));
    c.continuityTol = s.getScalarOr("continuityTol", c.continuityTol);
    c.pcorrTol = s.getScalarOr("pcorrTol", c.pcorrTol);
    c.momentumTol = s.getScalarOr("momentumTol", c.momentumTol);
    c.relaxU = s.getScalarOr("relaxU", c.relaxU);
    c.relaxP = s.getScalarOr("relaxP", c.relaxP);
    c.pRelaxStart = s.getScalarOr("pRelaxStart", c.pRelaxStart);
    c.nonOrthCorrectors = static_cast<int>(s.getScalarOr("nonOrthCorrectors", c.nonOrthCorrectors));
    c.linearTol = s.getScalarOr("linearTol", c.linearTol);
    c.linearMaxIter = static_cast<int>(s.getScalarOr("linearMaxIter", c.linearMaxIter));
    return c;
}

NetworkPipe resistor(const std::string& name, const std::string& from, const std::string& to, double r)
{
    // a pipe whose only law is its coefficient: dp = r q
    NetworkPipe p;
    p.name = name;
    p.fromName = from;
    p.toName = to;
    p.length = 10.0;
    p.diameter = 0.05;
    p.coupledResistance = r;
    return p;
}

} // namespace

int main(int argc, char** argv)
{
#ifdef CFG_ADAPTER
    const int need = 4;
#else
    const int need = 3;
#endif
    if (argc < need)
    {
        std::cerr << "usage: " << argv[0] << " <case.dict> <out>"
#ifdef CFG_ADAPTER
                  << " <single|batch>"
#endif
                  << "\n";
        return 2;
    }
    try
    {
        const std::string casePath = argv[1], out = argv[2];
        const Dictionary caseDict = Dictionary::parseFile(casePath);
        const Dictionary& nd = caseDict.getDict("network");
        OneDNetwork net;
        net.fluid = FluidProperties{nd.getScalar("rho"), nd.getScalar("mu")};
        for (const char* n : {"Src", "J1", "J2", "Snk"}) net.addNode(n);
        net.setNodeRate("Src", nd.getScalar("qIn"));
        net.setNodePressure("Snk", nd.getScalar("pOut"));
        net.addPipe(resistor("In", "Src", "J1", nd.getScalar("rIn")));
        net.addPipe(resistor("Out", "J2", "Snk", nd.getScalar("rOut")));

        const Schemes schemes = loadSchemes(caseDict);
        const SimpleControls ctl = controlsOf(caseDict);
        const Dictionary& bd = caseDict.getDict("blocks");
        std::vector<label> edges;
#ifdef CFG_ADAPTER
        std::vector<std::unique_ptr<gpu::GpuDetailBlock>> owned;
#else
        std::vector<std::unique_ptr<coupling::DetailBlock>> owned;
#endif
        std::vector<coupling::ICoupledElement*> partners;
        for (const std::string& name : bd.keys())
        {
            const Dictionary& b = bd.getDict(name);
            edges.push_back(net.addPipe(resistor(name, "J1", "J2", b.getScalar("resistance"))));
            polyMesh mesh = MeshLoader::fromCase(b, casePath);
            const TurbulenceConfig turb = TurbulenceConfig::fromCase(b);
            const scalar nu = b.getScalar("nu"), rho = b.getScalar("rho");
            const std::string shape = b.getWordOr("shape", "flat");
#ifdef CFG_ADAPTER
            owned.push_back(std::make_unique<gpu::GpuDetailBlock>(std::move(mesh), nu, rho, schemes, ctl, turb, shape));
#else
            owned.push_back(std::make_unique<coupling::DetailBlock>(std::move(mesh), nu, rho, schemes, ctl, -1e300,
                                                                    1e300, turb, shape));
#endif
            partners.push_back(owned.back().get());
        }

        const Dictionary& cd = caseDict.getDict("coupling");
        coupling::CoupledControls cc;
        cc.maxOuterIterations = static_cast<label>(cd.getScalarOr("maxOuterIterations", cc.maxOuterIterations));
        cc.relax = cd.getScalarOr("relax", cc.relax);
        cc.tolerance = cd.getScalarOr("tolerance", cc.tolerance);
        cc.accelerate = cd.getWordOr("accelerate", "no") == "yes";
        SteadyControls netCtl;
        netCtl.maxIter = 200;
        netCtl.tol = cd.getScalarOr("networkTol", 1e-10);

#ifdef CFG_ADAPTER
        std::unique_ptr<gpu::GpuDetailBlockBatch> batch;
        if (std::string(argv[3]) == "batch")
        {
            std::vector<gpu::GpuDetailBlock*> raw;
            for (auto& b : owned) raw.push_back(b.get());
            batch = std::make_unique<gpu::GpuDetailBlockBatch>(raw, net, edges, netCtl);
            partners = batch->elements();
        }
        else if (std::string(argv[3]) != "single")
        {
            std::cerr << "unknown partner mode " << argv[3] << "\n";
            return 2;
        }
#endif
        const coupling::CoupledResult res = coupling::solveCoupled1d3d(net, edges, partners, cc, netCtl);

        std::ofstream h(out + "/history.txt");
        h << std::setprecision(17);
        for (const auto& step : res.history)
            for (std::size_t i = 0; i < step.edges.size(); ++i)
            {
                const auto& e = step.edges[i];
                h << step.iteration << " " << i << " " << e.q << " " << e.dpPa << " " << e.resistance << " "
                  << e.sweeps << " " << (e.blockConverged ? 1 : 0) << "\n";
            }
        h << "result " << res.iterations << " " << (res.converged ? 1 : 0) << " " << res.residual << "\n";
#ifdef CFG_ADAPTER
        if (batch)
        {
            std::ofstream b(out + "/batch.txt");
            b << batch->batchedPasses() << " " << batch->singleRequests() << "\n";
        }
#endif
        return 0;
    }
    catch (const std::exception& e)
    {
        std::cerr << argv[0] << ": " << e.what() << "\n";
        return 1;
    }
}
