// osprey_dpd_glue.cpp -- reference-side binding of the B200 engine into
// CSimBox::Evolve; see osprey_dpd_glue.h.  Compiled against the reference's
// headers (its src directory on the include path) and linked with
// libospreydpd_cuda.so; every reference type is used through its public
// interface only.
#include "StdAfx.h"
#include "SimDefs.h"

#include "SimBox.h"
#include "ISimBox.h"
#include "IGlobalSimBox.h"
#include "CNTCell.h"
#include "AbstractBead.h"
#include "Bond.h"
#include "BondPair.h"
#include "LogSimErrorTrace.h"
#include "ccStopNoSave.h"

#include "osprey_dpd_glue.h"
#include "dpd_engine.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

namespace {

struct Glue {
    dpd_engine* eng = nullptr;
    bool failed = false;                 // creation or upload failed: the run was stopped
    std::vector<CAbstractBead*> beads;   // upload order: bead id order
    int32_t ntypes = 0;
    double dt = 0.0;
    std::vector<double> a, g;            // a_ij, gamma_ij last given to the engine
    std::vector<double> x, u, v, f, st;  // download buffers, 3 (9) per bead
    std::vector<int32_t> cell;
};

Glue& glue()
{
    static Glue g;
    return g;
}

// A fatal condition: logged and the run stopped, as the reference does for
// its own fatal errors (SimBox.cpp:442-443).
void stop_run(CSimBox* box, long t, const std::string& msg)
{
    new CLogSimErrorTrace(t, ("B200 engine: " + msg).c_str());
    box->AddCommandToFront(new ccStopNoSave(t + 1));
}

std::string engine_error(dpd_engine* e, const char* what, int rc)
{
    char buf[64];
    snprintf(buf, sizeof buf, " failed (%d): ", rc);
    return std::string(what) + buf + (e ? dpd_engine_last_error(e) : "");
}

// The reference's pair tables as the engine takes them (row-major T x T).
void pair_tables(const ISimBox* ib, int32_t T, std::vector<double>& a, std::vector<double>& g)
{
    a.assign((size_t)T * T, 0.0);
    g.assign((size_t)T * T, 0.0);
    for (int32_t i = 0; i < T; ++i)
        for (int32_t j = 0; j < T; ++j) {
            a[(size_t)i * T + j] = ib->GetDPDBeadConsInt(i, j);
            g[(size_t)i * T + j] = ib->GetDPDBeadDissInt(i, j);
        }
}

// Optional host-side corruption of one uploaded bead (OSPREY_DPD_GLUE_INJECT).
void inject(std::vector<double>& v3, std::vector<double>& f3, const std::vector<int64_t>& id)
{
    const char* spec = getenv("OSPREY_DPD_GLUE_INJECT");
    if (!spec) return;
    const char* colon = strchr(spec, ':');
    if (!colon) return;
    const long long target = atoll(colon + 1);
    for (size_t k = 0; k < id.size(); ++k)
        if (id[k] == target) {
            if (!strncmp(spec, "nan", 3)) v3[3 * k] = std::nan("");
            else if (!strncmp(spec, "force", 5)) f3[3 * k] = 1e308;
        }
}

bool create(CSimBox* box, long t)
{
    Glue& G = glue();
    const ISimBox* ib = box->GetISimBox();
    G.ntypes = (int32_t)ib->GetBeadTypeTotal();
    pair_tables(ib, G.ntypes, G.a, G.g);
    G.dt = ib->GetStepSize();
    dpd_params p{};
    p.nx = (int32_t)ib->GetCNTXCellNo();
    p.ny = (int32_t)ib->GetCNTYCellNo();
    p.nz = (int32_t)ib->GetCNTZCellNo();
    p.wx = ib->GetCNTXCellWidth();
    p.wy = ib->GetCNTYCellWidth();
    p.wz = ib->GetCNTZCellWidth();
    p.dt = G.dt;
    p.lambda = ib->GetLambda();
    p.kT = ib->GetTemperature();
    p.ntypes = G.ntypes;
    p.a = G.a.data();
    p.gamma = G.g.data();
    p.seed = (uint64_t)std::labs(ib->GetRNGSeed());
    const char* prec = getenv("OSPREY_DPD_PRECISION");
    p.precision = (prec && !strcmp(prec, "fp64")) ? DPD_PRECISION_FP64 : DPD_PRECISION_MIXED;
    const char* dev = getenv("OSPREY_DPD_DEVICE");
    p.device = dev ? atoi(dev) : -1;
    int rc = dpd_engine_create(&p, &G.eng);
    if (rc != DPD_OK) {
        G.eng = nullptr;
        stop_run(box, t, engine_error(nullptr, "dpd_engine_create", rc));
        return false;
    }
    // the beads of the CNT cells (CSimBox::GetAllBeadsInCNTCells), in id order
    AbstractBeadVector all = box->GetAllBeadsInCNTCells();
    G.beads.assign(all.begin(), all.end());
    std::sort(G.beads.begin(), G.beads.end(),
              [](const CAbstractBead* l, const CAbstractBead* r) { return l->GetId() < r->GetId(); });
    const size_t n = G.beads.size();
    std::vector<int64_t> id(n);
    std::vector<int32_t> type(n);
    std::vector<uint8_t> movable(n);
    std::vector<double> x3(3 * n), u3(3 * n), v3(3 * n), f3(3 * n);
    std::map<const CAbstractBead*, int64_t> idOf;
    for (size_t k = 0; k < n; ++k) {
        const CAbstractBead* b = G.beads[k];
        id[k] = b->GetId();
        type[k] = (int32_t)b->GetType();
        movable[k] = b->GetFrozen() ? 0 : 1;
        const double xs[3] = {b->GetXPos(), b->GetYPos(), b->GetZPos()};
        const double us[3] = {b->GetunPBCXPos(), b->GetunPBCYPos(), b->GetunPBCZPos()};
        const double vs[3] = {b->GetXMom(), b->GetYMom(), b->GetZMom()};
        const double fs[3] = {b->GetXForce(), b->GetYForce(), b->GetZForce()};
        for (int d = 0; d < 3; ++d) {
            x3[3 * k + d] = xs[d];
            u3[3 * k + d] = us[d];
            v3[3 * k + d] = vs[d];
            f3[3 * k + d] = fs[d];
        }
        idOf[b] = id[k];
    }
    inject(v3, f3, id);
    rc = dpd_engine_upload_beads(G.eng, (int64_t)n, id.data(), type.data(), movable.data(), x3.data(), u3.data(),
                                 v3.data(), f3.data());
    if (rc != DPD_OK) {
        stop_run(box, t, engine_error(G.eng, "dpd_engine_upload_beads", rc));
        return false;
    }
    // bonds and bond pairs of the polymers (CBond / CBondPair objects)
    const BondVector& bonds = ib->GetBonds();
    const BondPairVector& pairs = ib->GetBondPairs();
    std::map<const CBond*, int64_t> bondIndex;
    std::vector<int64_t> bh(bonds.size()), bt(bonds.size());
    std::vector<double> k2(bonds.size()), l0(bonds.size());
    for (size_t i = 0; i < bonds.size(); ++i) {
        bondIndex[bonds[i]] = (int64_t)i;
        bh[i] = bonds[i]->GetHead()->GetId();
        bt[i] = bonds[i]->GetTail()->GetId();
        k2[i] = bonds[i]->GetSprConst();
        l0[i] = bonds[i]->GetUnStrLength();
    }
    std::vector<int64_t> af(pairs.size()), as(pairs.size());
    std::vector<double> k3(pairs.size()), phi0(pairs.size());
    for (size_t i = 0; i < pairs.size(); ++i) {
        af[i] = bondIndex[pairs[i]->GetFirst()];
        as[i] = bondIndex[pairs[i]->GetSecond()];
        k3[i] = pairs[i]->GetModulus();
        phi0[i] = pairs[i]->GetPhi0();
    }
    rc = dpd_engine_upload_topology(G.eng, (int64_t)bonds.size(), bh.data(), bt.data(), k2.data(), l0.data(),
                                    (int64_t)pairs.size(), af.data(), as.data(), k3.data(), phi0.data());
    if (rc != DPD_OK) {
        stop_run(box, t, engine_error(G.eng, "dpd_engine_upload_topology", rc));
        return false;
    }
    G.x.resize(3 * n);
    G.u.resize(3 * n);
    G.v.resize(3 * n);
    G.f.resize(3 * n);
    G.st.resize(9 * n);
    G.cell.resize(n);
    return true;
}

// Commands between steps may change dt (SetTimeStepSize) or the pair tables
// (SetDPDBeadConsInt/DissInt): forward what changed.
int push_changes(CSimBox* box)
{
    Glue& G = glue();
    const ISimBox* ib = box->GetISimBox();
    const double dt = ib->GetStepSize();
    if (dt != G.dt) {
        G.dt = dt;
        const int rc = dpd_engine_set_dt(G.eng, dt);
        if (rc != DPD_OK) return rc;
    }
    std::vector<double> a, g;
    pair_tables(ib, G.ntypes, a, g);
    if (a != G.a || g != G.g) {
        G.a.swap(a);
        G.g.swap(g);
        return dpd_engine_set_pair_params(G.eng, G.ntypes, G.a.data(), G.g.data());
    }
    return DPD_OK;
}

// The engine's state into the bead objects, and the CNT cell lists rebuilt
// from the engine's cells.
int sync_beads(CSimBox* box)
{
    Glue& G = glue();
    int rc = dpd_engine_download(G.eng, G.x.data(), G.u.data(), G.v.data(), G.f.data(), G.st.data());
    if (rc == DPD_OK) rc = dpd_engine_cells(G.eng, G.cell.data());
    if (rc != DPD_OK) return rc;
    const size_t n = G.beads.size();
    for (size_t k = 0; k < n; ++k) {
        CAbstractBead* b = G.beads[k];
        b->SetXPos(G.x[3 * k]);
        b->SetYPos(G.x[3 * k + 1]);
        b->SetZPos(G.x[3 * k + 2]);
        b->SetunPBCXPos(G.u[3 * k]);
        b->SetunPBCYPos(G.u[3 * k + 1]);
        b->SetunPBCZPos(G.u[3 * k + 2]);
        b->SetXMom(G.v[3 * k]);
        b->SetYMom(G.v[3 * k + 1]);
        b->SetZMom(G.v[3 * k + 2]);
        b->SetXForce(G.f[3 * k]);
        b->SetYForce(G.f[3 * k + 1]);
        b->SetZForce(G.f[3 * k + 2]);
    }
    const CNTCellVector& cells = box->GetCNTCells();
    for (CCNTCell* c : cells) c->RemoveAllBeadsFromCell();
    for (size_t k = 0; k < n; ++k) {
        const int32_t c = G.cell[k];
        if (c < 0 || (size_t)c >= cells.size()) return DPD_E_STATE;
        cells[(size_t)c]->AddBeadtoCell(G.beads[k]);
    }
    return DPD_OK;
}

}  // namespace

bool OspreyDpdEvolve(CSimBox* box, long simTime, bool sync, bool renorm, OspreyDpdSync* out)
{
    Glue& G = glue();
    if (out) {
        out->stress9 = nullptr;
        out->beads = nullptr;
    }
    if (G.failed) return true;   // the run is being stopped; the reference state is left as it was
    if (!G.eng && !create(box, simTime)) {
        G.failed = true;
        return true;
    }
    int rc = push_changes(box);
    if (rc == DPD_OK && renorm) rc = dpd_engine_renormalise_mom(G.eng);
    if (rc == DPD_OK) rc = dpd_engine_step(G.eng, simTime, 1);
    if (rc == DPD_OK && sync) {
        rc = sync_beads(box);
        if (rc == DPD_OK && out) {
            out->stress9 = G.st.data();
            out->beads = &G.beads;
        }
    }
    if (rc != DPD_OK) {
        stop_run(box, simTime, engine_error(G.eng, "step", rc));
        G.failed = true;
    }
    return true;
}
