// ref_driver.cpp -- test harness around the UNMODIFIED Osprey-DPD reference.
//
// This file is test infrastructure (it pins the oracle to the reference), never part of the engine.
// It is linked against the reference's own objects, compiled from the
// reference's src/*.cpp by oracle/Makefile, and drives the reference through
// its public classes exactly as CSimulation::Initialize/Run do
// (Simulation.cpp:338-490):
//
//   CInputData(runId) -> GetInputData("dmpci."+runId)   (InputData.h:53,73)
//   CSimState(inputData) -> Assemble()                  (SimState.h:40,48)
//   [optional] overwrite bead state through the public setters
//              (AbstractBead.h:185-215)                 <- state injection
//   ISimBox::Instance(simState) -> Run()                (ISimBox.cpp:44, ISimBox.h:176)
//
// --rng-seed S restarts the reference's pair-noise LCG at |S| through its
// public CCNTCell::SetRNGSeed (CNTCell.cpp:134-137) just before Run(), so the
// draws consumed by the initial-state builder do not matter.
//
// Run() is the reference's own step loop (SimBox.cpp:1272-1355) calling
// Evolve() (SimBox.cpp:977-1120) every step; it is timed on its own so the
// reported bead-steps/s exclude parsing, building and the bead binning.
//
// Usage (run inside the directory that holds dmpci.<runId>):
//   osprey_ref_driver <runId> [--inject state.bin] [--topology topo.bin]
//                             [--dump out.bin] [--rng-seed S] [--dump-initial init.bin]
//                             [--paraview 1]
// Prints one JSON line: {"beads":N,"steps":T,"run_seconds":s,...}
//
// Binary formats (little endian):
//   state.bin : "DPDSTATE" int64 n, then n records ordered by bead id:
//               int64 id, int64 type, double x[3], unpbc[3], v[3], f[3]
//   topo.bin  : "DPDTOPO1" int64 nb, nb x {int64 head_id, tail_id; double k2, l0}
//               int64 na, na x {int64 first_bond, second_bond; double k3, phi0}
//               (bond indices refer to the bond order written here, which is
//               the reference's own polymer-by-polymer order, InitialState.cpp:498-505)
//   out.bin   : "DPDDUMP1" int64 n, int64 steps, then n records by bead id:
//               int64 id, int64 type, double x[3], unpbc[3], v[3], f[3], stress[9]
//   slices    : (--slices f --slice-dims S,T,NBT,NBPT) "DPDSLICE" int64 S, T, NBT,
//               NBPT, nb, na; then the slice stress of the last step through
//               CMonitor's public getters (Monitor.h:248-276): double
//               pair[S][T*T][9], bond[S][NBT][9], bondpair[S][NBPT][9]; then
//               int64 type of every bond and bond pair (CBond/CBondPair::GetType)

#include "StdAfx.h"
#include "SimDefs.h"

#include "CurrentState.h"
#include "ParaviewFormat.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

// Per-bead stress (AbstractBead.h:258) has no public getter.  The harness
// reads it by widening access for this translation unit only; member order
// and therefore the object layout are unchanged.
#define protected public
#include "AbstractBead.h"
#undef protected

#include "InputData.h"
#include "SimState.h"
#include "ISimBox.h"
#include "Bead.h"
#include "Bond.h"
#include "BondPair.h"
#include "CNTCell.h"
#include "Monitor.h"

namespace {

struct BeadRec {
    long long id, type;
    double x[3], u[3], v[3], f[3];
};

bool read_exact(FILE* fp, void* p, size_t n) { return fread(p, 1, n, fp) == n; }

int fail(const char* msg) {
    fprintf(stderr, "osprey_ref_driver: %s\n", msg);
    return 2;
}

}  // namespace

// out.bin format (see the header comment), beads by id.
static bool write_dump(const char* path, const std::vector<CBead*>& byId, long n, long steps)
{
    FILE* fp = fopen(path, "wb");
    if (!fp) return false;
    fwrite("DPDDUMP1", 1, 8, fp);
    long long nn = n, ss = steps;
    fwrite(&nn, 8, 1, fp);
    fwrite(&ss, 8, 1, fp);
    for (long id = 1; id <= n; ++id) {
        const CBead* b = byId[id];
        long long it[2] = {b->GetId(), b->GetType()};
        double d[21] = {b->GetXPos(), b->GetYPos(), b->GetZPos(),
                        b->GetunPBCXPos(), b->GetunPBCYPos(), b->GetunPBCZPos(),
                        b->GetXMom(), b->GetYMom(), b->GetZMom(),
                        b->GetXForce(), b->GetYForce(), b->GetZForce()};
        for (int k = 0; k < 9; ++k) d[12 + k] = b->m_Stress[k];
        fwrite(it, 8, 2, fp);
        fwrite(d, 8, 21, fp);
    }
    fclose(fp);
    return true;
}

int main(int argc, char** argv)
{
    if (argc < 2) return fail("usage: osprey_ref_driver <runId> [--inject f] [--topology f] [--dump f]");
    const zString runId = argv[1];
    const char* injectPath = 0;
    const char* topoPath = 0;
    const char* dumpPath = 0;
    const char* rngSeed = 0;
    const char* slicePath = 0;
    const char* sliceDims = 0;
    const char* initialPath = 0;
    bool paraview = false;
    for (int a = 2; a + 1 < argc; a += 2) {
        if (!strcmp(argv[a], "--inject")) injectPath = argv[a + 1];
        else if (!strcmp(argv[a], "--topology")) topoPath = argv[a + 1];
        else if (!strcmp(argv[a], "--dump")) dumpPath = argv[a + 1];
        else if (!strcmp(argv[a], "--rng-seed")) rngSeed = argv[a + 1];
        else if (!strcmp(argv[a], "--slices")) slicePath = argv[a + 1];
        else if (!strcmp(argv[a], "--slice-dims")) sliceDims = argv[a + 1];
        else if (!strcmp(argv[a], "--dump-initial")) initialPath = argv[a + 1];
        else if (!strcmp(argv[a], "--paraview")) paraview = atoi(argv[a + 1]) != 0;
        else return fail("unknown option");
    }

    auto tSetup0 = std::chrono::steady_clock::now();
    CInputData* pIn = new CInputData(runId);
    if (!pIn->GetInputData(xxBase::GetCDFPrefix() + runId)) return fail("dmpci rejected by CInputData");
    CSimState* pState = new CSimState(*pIn);
    if (!pState->Assemble()) return fail("CSimState::Assemble failed");

    const BeadVector& beads = pState->GetInitialStateBeads();
    const long n = static_cast<long>(beads.size());

    // Map bead id -> bead (ids are 1..N assigned in polymer order, InitialState.cpp:490-500).
    std::vector<CBead*> byId(n + 1, static_cast<CBead*>(0));
    for (long i = 0; i < n; ++i) {
        const long id = beads[i]->GetId();
        if (id < 1 || id > n || byId[id]) return fail("unexpected bead id layout");
        byId[id] = beads[i];
    }

    // The builder's output (CSimState::Assemble -> CInitialState -> e.g.
    // CRandomBuilder::Assemble, RandomBuilder.cpp:71-361), before any
    // injection or step: the dump format with steps = 0.
    if (initialPath && !write_dump(initialPath, byId, n, 0)) return fail("cannot write initial dump");

    if (injectPath) {
        FILE* fp = fopen(injectPath, "rb");
        if (!fp) return fail("cannot open inject file");
        char magic[8];
        long long nin = 0;
        if (!read_exact(fp, magic, 8) || memcmp(magic, "DPDSTATE", 8) || !read_exact(fp, &nin, 8))
            return fail("bad inject header");
        if (nin != n) return fail("inject bead count differs from the dmpci's bead count");
        for (long k = 0; k < n; ++k) {
            BeadRec r;
            if (!read_exact(fp, &r, sizeof r)) return fail("short inject file");
            if (r.id < 1 || r.id > n) return fail("inject id out of range");
            CBead* b = byId[r.id];
            if (b->GetType() != r.type) return fail("inject type differs from the dmpci's bead type");
            b->SetXPos(r.x[0]); b->SetYPos(r.x[1]); b->SetZPos(r.x[2]);
            b->SetunPBCXPos(r.u[0]); b->SetunPBCYPos(r.u[1]); b->SetunPBCZPos(r.u[2]);
            b->SetInitialXPos(r.u[0]); b->SetInitialYPos(r.u[1]); b->SetInitialZPos(r.u[2]);
            b->SetXMom(r.v[0]); b->SetYMom(r.v[1]); b->SetZMom(r.v[2]);
            b->SetXForce(r.f[0]); b->SetYForce(r.f[1]); b->SetZForce(r.f[2]);
        }
        fclose(fp);
    }

    if (topoPath) {
        const BondVector& bonds = pState->GetBonds();
        const BondPairVector& pairs = pState->GetBondPairs();
        std::map<const CBond*, long long> bondIndex;
        for (size_t i = 0; i < bonds.size(); ++i) bondIndex[bonds[i]] = static_cast<long long>(i);
        FILE* fp = fopen(topoPath, "wb");
        if (!fp) return fail("cannot open topology file");
        fwrite("DPDTOPO1", 1, 8, fp);
        long long nb = static_cast<long long>(bonds.size());
        fwrite(&nb, 8, 1, fp);
        for (size_t i = 0; i < bonds.size(); ++i) {
            long long ht[2] = {bonds[i]->GetHead()->GetId(), bonds[i]->GetTail()->GetId()};
            double kl[2] = {bonds[i]->GetSprConst(), bonds[i]->GetUnStrLength()};
            fwrite(ht, 8, 2, fp);
            fwrite(kl, 8, 2, fp);
        }
        long long na = static_cast<long long>(pairs.size());
        fwrite(&na, 8, 1, fp);
        for (size_t i = 0; i < pairs.size(); ++i) {
            long long fs[2] = {bondIndex[pairs[i]->GetFirst()], bondIndex[pairs[i]->GetSecond()]};
            double kp[2] = {pairs[i]->GetModulus(), pairs[i]->GetPhi0()};
            fwrite(fs, 8, 2, fp);
            fwrite(kp, 8, 2, fp);
        }
        fclose(fp);
    }

    ISimBox* pBox = ISimBox::Instance(*pState);
    if (rngSeed) CCNTCell::SetRNGSeed(atol(rngSeed));
    const long steps = pBox->GetTotalTime();
    auto tRun0 = std::chrono::steady_clock::now();
    pBox->Run();
    auto tRun1 = std::chrono::steady_clock::now();

    if (dumpPath && !write_dump(dumpPath, byId, n, steps)) return fail("cannot open dump file");

    // --paraview 1: the reference's own Paraview snapshot of the final state
    // (CCurrentState + CParaviewFormat, CurrentState.cpp:109-244,
    // ParaviewFormat.cpp:72-112), written as dmpccs.<runId>.con.<steps>.vtk
    if (paraview) {
        CParaviewFormat* pFormat = new CParaviewFormat(pBox->GetSimSpaceXLength(), pBox->GetSimSpaceYLength(),
                                                       pBox->GetSimSpaceZLength(), false, pBox->GetBeadTypeTotal());
        CCurrentState cs(steps, runId, pBox, pFormat, false, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0);
        if (!cs.Serialize()) return fail("CCurrentState::Serialize failed");
    }

    if (slicePath) {
        long long dims[4] = {0, 0, 0, 0};
        if (!sliceDims || sscanf(sliceDims, "%lld,%lld,%lld,%lld", &dims[0], &dims[1], &dims[2], &dims[3]) != 4)
            return fail("--slices needs --slice-dims S,T,NBT,NBPT");
        const CMonitor* mon = pBox->GetMonitor();
        FILE* fp = fopen(slicePath, "wb");
        if (!fp) return fail("cannot open slice file");
        const BondVector& bonds = pState->GetBonds();
        const BondPairVector& bps = pState->GetBondPairs();
        long long hdr[6] = {dims[0], dims[1], dims[2], dims[3], (long long)bonds.size(), (long long)bps.size()};
        fwrite("DPDSLICE", 1, 8, fp);
        fwrite(hdr, 8, 6, fp);
        for (long sl = 0; sl < dims[0]; ++sl)
            for (long k = 0; k < dims[1] * dims[1]; ++k) {
                const double q[9] = {mon->GetSliceStress11(sl, k), mon->GetSliceStress12(sl, k),
                                     mon->GetSliceStress13(sl, k), mon->GetSliceStress21(sl, k),
                                     mon->GetSliceStress22(sl, k), mon->GetSliceStress23(sl, k),
                                     mon->GetSliceStress31(sl, k), mon->GetSliceStress32(sl, k),
                                     mon->GetSliceStress33(sl, k)};
                fwrite(q, 8, 9, fp);
            }
        for (long sl = 0; sl < dims[0]; ++sl)
            for (long k = 0; k < dims[2]; ++k) {
                const double q[9] = {mon->GetSliceStressBond11(sl, k), mon->GetSliceStressBond12(sl, k),
                                     mon->GetSliceStressBond13(sl, k), mon->GetSliceStressBond21(sl, k),
                                     mon->GetSliceStressBond22(sl, k), mon->GetSliceStressBond23(sl, k),
                                     mon->GetSliceStressBond31(sl, k), mon->GetSliceStressBond32(sl, k),
                                     mon->GetSliceStressBond33(sl, k)};
                fwrite(q, 8, 9, fp);
            }
        for (long sl = 0; sl < dims[0]; ++sl)
            for (long k = 0; k < dims[3]; ++k) {
                const double q[9] = {mon->GetSliceStressBondPair11(sl, k), mon->GetSliceStressBondPair12(sl, k),
                                     mon->GetSliceStressBondPair13(sl, k), mon->GetSliceStressBondPair21(sl, k),
                                     mon->GetSliceStressBondPair22(sl, k), mon->GetSliceStressBondPair23(sl, k),
                                     mon->GetSliceStressBondPair31(sl, k), mon->GetSliceStressBondPair32(sl, k),
                                     mon->GetSliceStressBondPair33(sl, k)};
                fwrite(q, 8, 9, fp);
            }
        for (size_t i = 0; i < bonds.size(); ++i) {
            const long long t = bonds[i]->GetType();
            fwrite(&t, 8, 1, fp);
        }
        for (size_t i = 0; i < bps.size(); ++i) {
            const long long t = bps[i]->GetType();
            fwrite(&t, 8, 1, fp);
        }
        fclose(fp);
    }

    const double setupS = std::chrono::duration<double>(tRun0 - tSetup0).count();
    const double runS = std::chrono::duration<double>(tRun1 - tRun0).count();
    printf("{\"beads\": %ld, \"steps\": %ld, \"bonds\": %ld, \"bondpairs\": %ld, "
           "\"setup_seconds\": %.6f, \"run_seconds\": %.6f, \"bead_steps_per_s\": %.6e}\n",
           n, steps, static_cast<long>(pState->GetBonds().size()),
           static_cast<long>(pState->GetBondPairs().size()), setupS, runS,
           runS > 0 ? static_cast<double>(n) * steps / runS : 0.0);
    return 0;
}
