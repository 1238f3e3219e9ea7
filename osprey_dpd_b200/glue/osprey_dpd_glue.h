// osprey_dpd_glue.h -- the reference-side binding of the B200 engine
// (libospreydpd_cuda.so, include/dpd_engine.h) into Osprey-DPD's
// CSimBox::Evolve (SimBox.cpp:977-1120).
//
// A build with OSPREY_DPD_CUDA compiles a copy of SimBox.cpp whose Evolve
// starts with
//
//     OspreyDpdSync sync = {0, 0};
//     if (OspreyDpdEvolve(this, m_SimTime, <sample, display or restart step, or the last>,
//                         <momentum renormalisation due>, &sync)) { <per-bead stress>; return; }
//
// (osprey_dpd_b200/glue/patch_simbox.py writes that copy), so the engine
// advances the step instead of the CNT-cell loops and every other part of the
// reference -- input files, builders, commands, CMonitor, analysis, output --
// runs unchanged.  The engine is created on the first call from the
// reference's own state (ISimBox getters: box, dt, lambda, kT, a_ij, gamma_ij,
// RNGSeed; the beads of the CNT cells; CBond / CBondPair objects).  On steps
// where the reference reads beads (Sample, SaveCurrentState,
// SaveRestartState, the last step) the bead objects receive x, unPBC, v, F
// and the CNT cell lists are rebuilt from the engine's cell assignment
// (CCNTCell::RemoveAllBeadsFromCell / AddBeadtoCell, CNTCell.cpp:2339-2357);
// the per-bead stress is written by the caller, a friend of CAbstractBead.
// Parameter changes made by commands between steps are forwarded: the time
// step (SetTimeStepSize) and the a_ij / gamma_ij tables
// (SetDPDBeadConsInt/DissInt).  A non-zero engine status stops the run as the
// reference stops on fatal errors (CLogSimErrorTrace + ccStopNoSave,
// SimBox.cpp:436-445).
//
// Environment: OSPREY_DPD_PRECISION=fp64 selects the all-FP64 engine (default
// mixed); OSPREY_DPD_DEVICE selects the CUDA device; OSPREY_DPD_GLUE_INJECT
// ("nan:<bead id>" or "force:<bead id>") corrupts one bead of the uploaded
// state on the host -- a non-finite velocity, which the upload rejects, or a
// 1e308 force, which the device step turns into a non-finite state -- to
// exercise the error path.
#pragma once

#include <vector>

class CSimBox;
class CAbstractBead;

struct OspreyDpdSync {
    const double* stress9;                       // 9 per bead, in the order of *beads (NULL: nothing to write)
    const std::vector<CAbstractBead*>* beads;
};

// Runs timestep simTime on the engine.  Returns true when the engine took the
// step (the caller skips the reference's own body), false when the engine is
// not in use.  sync: copy the state back into the bead objects after the
// step.  renorm: CSimBox::UpdateRenormalisedMom is due before this step.
bool OspreyDpdEvolve(CSimBox* box, long simTime, bool sync, bool renorm, OspreyDpdSync* out);
