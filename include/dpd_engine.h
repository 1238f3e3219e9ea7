/* dpd_engine.h -- C ABI of the B200 DPD step engine (libospreydpd_cuda.so).
 *
 * The engine replaces the body of Osprey-DPD's per-timestep loop,
 * CSimBox::Evolve (SimBox.cpp:977-1120), i.e.
 *   CCNTCell::UpdatePos    (CNTCell.cpp:1598-2262)
 *   CCNTCell::UpdateForce  (CNTCell.cpp:877-1572, DPD branch 1103-1572)
 *   CSimBox::AddBondForces / CBond::AddForce            (SimBox.cpp:1382-1417, Bond.cpp:111-162)
 *   CSimBox::AddBondPairForces / CBondPair::AddForce    (SimBox.cpp:1423-1439, BondPair.cpp:138-286)
 *   CCNTCell::UpdateMom    (CNTCell.cpp:2280-2310)
 *   CSimBox::CNTCellCheck  (SimBox.cpp:1365-1371, CNTCell.cpp:2628-2700)
 * plus the single-bead sums of CMonitor::CalculateSingleBeadData
 * (Monitor.cpp:790-1040) that the host needs on sample steps.
 *
 * Conventions: plain pointers and sizes, no CUDA or C++ types.  Every call
 * returns 0 on success or a negative DPD_E* code; dpd_engine_last_error()
 * gives the message.  Host arrays are in bead-upload order (the reference's
 * bead-vector order, i.e. bead id order), xyz interleaved ("x3" = n*3).
 * One CUDA stream per engine; calls on one engine are not re-entrant.
 * The reference has no FFI of its own: the entry points below are the seam of
 * the CSimBox/CCNTCell/CBond/CBondPair classes, one call per responsibility.
 */
#ifndef DPD_ENGINE_H
#define DPD_ENGINE_H

#include <stdint.h>

#if defined(__GNUC__)
#define DPD_API __attribute__((visibility("default")))
#else
#define DPD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define DPD_OK                 0
#define DPD_E_ARG             -1   /* invalid argument                       */
#define DPD_E_CUDA            -2   /* CUDA runtime error                     */
#define DPD_E_STATE           -3   /* call out of order (e.g. step before upload) */
#define DPD_E_BOX             -4   /* bead outside the box at upload          */
#define DPD_E_STATUS          -5   /* device status word reported a fatal condition */
#define DPD_E_NOMEM           -6   /* host or device allocation failed       */
#define DPD_E_LIMIT           -7   /* system larger than a fixed-size buffer allows */

#define DPD_PRECISION_MIXED    0   /* FP32 pair/bond forces, FP64 x, v and sums */
#define DPD_PRECISION_FP64     1   /* everything FP64                          */

/* Device status bits, OR-ed by the kernels (dpd_engine_status). */
#define DPD_STATUS_CELL_SKIP      0x1u  /* a bead is filed in a cell other than floor(x/w):
                                            it moved more than one cell in a step (the
                                            reference logs CLogCNTBeadError, CNTCell.cpp:2650) */
#define DPD_STATUS_NONFINITE      0x2u  /* a non-finite position, velocity or force       */
#define DPD_STATUS_IMAGE_OVERFLOW 0x4u  /* a periodic image counter left +-511 box lengths */
#define DPD_STATUS_INTERNAL       0x8u  /* an internal capacity check tripped (a bug): results invalid */
#define DPD_STATUS_SLAB_REACH     0x10u /* a slab's owned bead lost a bond or bond pair: its partner
                                           lies beyond the ghost layers (dpd_engine_slab_*)      */
#define DPD_STATUS_FATAL_MASK     (DPD_STATUS_NONFINITE | DPD_STATUS_IMAGE_OVERFLOW | DPD_STATUS_INTERNAL | \
                                   DPD_STATUS_SLAB_REACH)

/* Kernel ids for dpd_engine_profile_read (the kernels of one step, in order). */
#define DPD_KERNEL_UPDATE_POS   0   /* UpdatePos drift + cell move             */
#define DPD_KERNEL_SCAN_CELLS   1   /* cell start offsets                      */
#define DPD_KERNEL_PERMUTE      2   /* arrival slot -> new slot                */
#define DPD_KERNEL_GATHER       3   /* cell-sorted state + force shadows       */
#define DPD_KERNEL_PAIR_FORCES  4   /* DPD pair forces (UpdateForce)           */
#define DPD_KERNEL_UPDATE_MOM   5   /* UpdateMom + single-bead sums            */
#define DPD_KERNEL_REDUCE_OBS   6   /* final FP64 sums                         */
#define DPD_KERNEL_DOWNLOAD     7   /* slot order -> bead order                */
#define DPD_KERNEL_KINETIC      8   /* kinetic sums without a step             */
#define DPD_KERNEL_BONDED       9   /* bond + bond-pair forces (FP64)          */
#define DPD_KERNEL_SLICES      10   /* slice stress profile, pair part (sample steps) */
#define DPD_NUM_KERNELS         11

typedef struct dpd_engine dpd_engine;

/* Parameters of CCNTCell::SetSimBoxLengths / SetTimeStepConstants /
 * SetDPDBeadStructure / SetRNGSeed (CNTCell.cpp:134-203, SimState.cpp:69-95). */
typedef struct dpd_params {
    int32_t nx, ny, nz;       /* CNT cells per axis; each >= 3                      */
    double  wx, wy, wz;       /* CNT cell widths; each >= 1 (the cut-off is 1)       */
    double  dt, lambda, kT;   /* Step, Lambda, Temp                                  */
    int32_t ntypes;           /* bead types, 1..32                                   */
    const double* a;          /* ntypes*ntypes a_ij, row-major, symmetric            */
    const double* gamma;      /* ntypes*ntypes gamma_ij                              */
    uint64_t seed;            /* pair-noise seed (|RNGSeed|)                          */
    int32_t precision;        /* DPD_PRECISION_*                                     */
    int32_t device;           /* CUDA device ordinal, or -1 for the current device   */
} dpd_params;

/* Single-bead sums of CMonitor::CalculateSingleBeadData (Monitor.cpp:790-1040),
 * accumulated in FP64 on the device at the end of the last dpd_engine_step. */
typedef struct dpd_obs {
    int64_t step;             /* m_SimTime of the state the sums describe             */
    int64_t n;
    double  sum_v[3];         /* sum of momenta (mass 1)                              */
    double  sum_v2[3];        /* sum of squared momenta per axis                      */
    double  virial[9];        /* sum of per-bead m_Stress (pair + bond), row-major    */
    double  sum_x[3];         /* sum of positions                                     */
    double  ang_mom[3];       /* sum of x cross v                                     */
    double  kT;               /* (sum v^2)/(3N)                    Monitor.cpp:979     */
    double  pressure;         /* (sum v^2 + trace virial)/(3V)     Monitor.cpp:981-982 */
    int32_t has_virial;       /* 0 if no step has run since upload                    */
    int32_t pad;
} dpd_obs;

/* One box of a replica batch: its CNT cells, widths, pair tables (ntypes of
 * the shared parameters) and pair-noise seed. */
typedef struct dpd_box {
    int32_t nx, ny, nz;
    double  wx, wy, wz;
    const double* a;
    const double* gamma;
    uint64_t seed;
} dpd_box;

/* Creates an engine for one box.  Replaces the CCNTCell statics set in
 * CSimState::CSimState (SimState.cpp:55-110). */
DPD_API int dpd_engine_create(const dpd_params* params, dpd_engine** out);

/* Copies the beads in (ownership stays with the caller).  Replaces
 * CSimBox::MakeCNTCells + AssignBeadstoCells (SimBox.cpp:715-877): beads are
 * binned with the reference's (long)(x/w) rule.  movable may be NULL (all
 * movable); unpbc3 may be NULL (= x3); f3 may be NULL (= 0). */
DPD_API int dpd_engine_upload_beads(dpd_engine* e, int64_t n, const int64_t* id, const int32_t* type,
                            const uint8_t* movable, const double* x3, const double* unpbc3,
                            const double* v3, const double* f3);

/* Builds the random initial state of CRandomBuilder::Assemble
 * (RandomBuilder.cpp:71-361, no walls, 3-d) on the device and uploads it as
 * dpd_engine_upload_beads would (unPBC = x, F = 0, all movable).  Replaces
 * the builder's loop over the beads in CInitialState (InitialState.cpp:
 * 451-520): id[i], type[i] are the i-th bead the reference creates; the
 * reference's generator (CCNTCell::Randf) starts at rng_seed (the |RNGSeed|
 * of the control file, CNTCell.cpp:134-137) and rng_skip draws are consumed
 * first (0 for the reference's random state); bond_head/bond_tail are bead
 * indices (0-based, into id) in the reference's polymer order, used for its
 * bond shortening.  kT is the engine's.  Positions equal the reference's bit
 * for bit; velocities agree to a few ulps (device acos/sin/cos, tree sums).
 * x3_out / v3_out (3 per bead, bead order) receive the built state when not
 * NULL.  Single-box engines only.  (Bond shortening moves a tail
 * coordinate to a point between the head's and its own, so every bead stays
 * in the box.)  The first call computes the reference's velocity-magnitude
 * table (CBuilder::MaxwellDist, max(n, 10^7) entries) on the host, about
 * half a second, and keeps it (8 bytes per entry) for the process. */
DPD_API int dpd_engine_build_random(dpd_engine* e, int64_t n, const int64_t* id, const int32_t* type,
                                    uint64_t rng_seed, int64_t rng_skip, int64_t nb, const int64_t* bond_head,
                                    const int64_t* bond_tail, double* x3_out, double* v3_out);

/* Builds the lamella initial state of CLamellaBuilder::Assemble
 * (LamellaBuilder.cpp:126-1010; no walls, no polymerised bonds) on the device
 * and uploads it as dpd_engine_upload_beads would (unPBC = x, F = 0, all
 * movable), with the in-plane Maxwell velocities of
 * CBuilder::AssignMaxwellVelocities (Builder.cpp:4207-4330).  Beads in the
 * reference's creation order (id, type); polymer p holds beads
 * [poly_first[p], poly_first[p+1]) (npoly + 1 entries) and has type
 * poly_type[p]; the bilayer is made of the polymers of type lipid_type, whose
 * head and tail beads sit at head_offset / tail_offset; normal 0, 1, 2 = x, y,
 * z; centre a fraction of the box length along the normal; thickness, straight
 * (linearise) or scattered chains, the upper monolayer's share as the
 * control file's State lamella block gives them.  The reference's generator
 * starts at rng_seed with rng_skip draws consumed first; bonds are bead
 * indices in polymer order (the other polymers' bonds are shortened as the
 * reference does).  Positions equal the reference's bit for bit; velocities
 * agree to a few ulps (device sin/cos, tree sums).  x3_out / v3_out receive
 * the built state when not NULL.  DPD_E_ARG when the bilayer or its lattice
 * does not fit the box. */
DPD_API int dpd_engine_build_lamella(dpd_engine* e, int64_t n, const int64_t* id, const int32_t* type,
                                     int64_t npoly, const int64_t* poly_first, const int32_t* poly_type,
                                     int32_t lipid_type, int32_t head_offset, int32_t tail_offset, int32_t normal,
                                     double centre, double thickness, int32_t linearise, double upper_fraction,
                                     uint64_t rng_seed, int64_t rng_skip, int64_t nb, const int64_t* bond_head,
                                     const int64_t* bond_tail, double* x3_out, double* v3_out);

/* Bonds (CBond: head id, tail id, k2, l0; Bond.h:45-52) and bond pairs
 * (CBondPair: indices of its first and second bond in this bond list, k3,
 * phi0 in radians; BondPair.h:23-30). */
DPD_API int dpd_engine_upload_topology(dpd_engine* e, int64_t nb, const int64_t* bond_head_id,
                               const int64_t* bond_tail_id, const double* k2, const double* l0,
                               int64_t na, const int64_t* first_bond, const int64_t* second_bond,
                               const double* k3, const double* phi0);

/* Replaces the whole a_ij / gamma_ij tables (CCNTCell::SetDPDBeadConsInt /
 * SetDPDBeadDissInt, CNTCell.cpp:434-456, and AddDPDBeadType, :498). */
DPD_API int dpd_engine_set_pair_params(dpd_engine* e, int32_t ntypes, const double* a, const double* gamma);

/* CCNTCell::ChangeTimeStepConstants (CNTCell.cpp:357): ignored unless dt > 0. */
DPD_API int dpd_engine_set_dt(dpd_engine* e, double dt);

/* CCNTCell::ToggleDPDBeadThermostat (CNTCell.cpp:318): on = 0 zeroes gamma
 * (dissipative and random forces), on = 1 restores it. */
DPD_API int dpd_engine_set_thermostat(dpd_engine* e, int32_t on);

/* CCNTCell::ToggleDPDBeadConservativeForces (CNTCell.cpp:235). */
DPD_API int dpd_engine_set_conservative(dpd_engine* e, int32_t on);

/* CSimBox::UpdateRenormalisedMom (SimBox.cpp:3177-3225), which the
 * reference's Run calls before Evolve when momentum renormalisation is on and
 * m_SimTime % period == 0 (SimBox.cpp:1314-1317): every bead's momentum is
 * divided by sqrt(sum v^2 / (3 N kT)), the sum taken in FP64 on the device.
 * Asynchronous (queued on the engine's stream).  Single-box engines; kT > 0. */
DPD_API int dpd_engine_renormalise_mom(dpd_engine* e);

/* Runs nsteps timesteps; first_step is the reference's m_SimTime of the first
 * (it keys the pair noise).  Asynchronous: returns once the work is queued,
 * without waiting for earlier calls.  The kernels of a call are captured once
 * as a CUDA graph per (step count, buffer parity, sample pattern, stream) and
 * replayed after that (DPD_GRAPHS=0 launches them one by one).  The
 * single-bead sums are taken at the end of the last step.
 * Returns the last device status without waiting: each call's first kernel
 * publishes the status word of all work queued before it to pinned host
 * memory, and the next call reads that word; if it holds a bit of
 * DPD_STATUS_FATAL_MASK the call returns DPD_E_STATUS (message in
 * dpd_engine_last_error) and queues nothing, so a fatal condition surfaces
 * at most two calls after the step that raised it (at once after
 * dpd_engine_status, download, cells or observables, which wait).  A new
 * bead upload clears the status. */
DPD_API int dpd_engine_step(dpd_engine* e, int64_t first_step, int32_t nsteps);

/* Steps at which the single-bead sums and the per-bead virial are taken:
 * period > 0 samples every step with m_SimTime % period == 0, the rule of
 * ISimState::TimeToSample (ISimState.cpp:468-471); period = 0 (the default)
 * samples at the last step of every dpd_engine_step call.  The virial costs
 * extra work, so other steps skip it as the reference's monitor does. */
DPD_API int dpd_engine_set_sample_period(dpd_engine* e, int64_t period);

/* Launch shape of the pair-force kernel (what the autotuner varies): hit-list
 * capacity per bead before a force pass (8..64, default 32), resident blocks
 * per SM of a persistent grid (0 = one 128-bead tile per block, the default),
 * preferred shared-memory carveout in percent (-1 = driver default). */
DPD_API int dpd_engine_set_launch_shape(dpd_engine* e, int32_t hitcap, int32_t persistent_blocks_per_sm,
                                        int32_t smem_carveout);

/* Pair-force scheme.  DPD_PAIR_FULL_SHELL (default): each bead sums its own
 * 27-cell neighbourhood; every pair is evaluated twice and the forces are
 * bitwise reproducible.  DPD_PAIR_HALF_SHELL: every pair once, over the
 * reference's own 13-cell half shell (CNTCell.cpp:1103-1572); the partner's
 * share is added with atomics, so the last bits of the FP32/FP64 force sums
 * vary from run to run, and the sampled pair virial goes whole to one bead of
 * the pair.  No counterpart in the reference's interface. */
#define DPD_PAIR_FULL_SHELL 0
#define DPD_PAIR_HALF_SHELL 1
/* DPD_PAIR_STAGED: the half-shell pair set with each 128-bead tile's
 * neighbour rows staged in shared memory; same accuracy and run-to-run
 * variation as DPD_PAIR_HALF_SHELL (slower on a B200: kept for comparison). */
#define DPD_PAIR_STAGED     2
DPD_API int dpd_engine_set_pair_scheme(dpd_engine* e, int32_t scheme);

/* Beads per block (tile) of the half-shell pair kernel: 64 (default, 0) or
 * 128, the same warps per SM either way; an autotuned axis. */
DPD_API int dpd_engine_set_pair_tile(dpd_engine* e, int32_t beads_per_block);

/* Waits for queued work; returns the device status bits seen so far. */
DPD_API int dpd_engine_status(dpd_engine* e, uint32_t* status_bits);

/* Copies the state out (synchronous); any pointer may be NULL.  stress9 is
 * the per-bead virial of the latest sample step (pair part split evenly
 * between the two beads of a pair; bond part on the head bead as
 * Bond.cpp:151-160), zero before any sample step. */
DPD_API int dpd_engine_download(dpd_engine* e, double* x3, double* unpbc3, double* v3, double* f3,
                        double* stress9);

/* Bead ids and types in upload order (n entries each; either may be NULL):
 * the caller's arrays as uploaded, or after dpd_engine_slab_unpack the
 * local box's beads as the exchange formed them. */
DPD_API int dpd_engine_bead_ids(dpd_engine* e, int64_t* id, int32_t* type);

/* Index of the CNT cell each bead is filed in (nx*(ny*iz+iy)+ix). */
DPD_API int dpd_engine_cells(dpd_engine* e, int32_t* cell);

/* Single-bead sums of the latest sample step (synchronous); before any sample
 * step since the upload, the kinetic sums of the current state without a
 * virial (has_virial = 0). */
DPD_API int dpd_engine_observables(dpd_engine* e, dpd_obs* out);

/* Slice stress profile of the reference's CMonitor (AddBeadStress,
 * AddBondStress, AddBondPairStress and ZeroSliceStress, Monitor.cpp:1900-2755;
 * read by the stress-profile analysis, aaStressTensor1d.cpp:150-200).  With
 * nslices > 0 every sample step splits each pair, bond and bond-pair
 * contribution (force x separation, 9 components) over nslices z slices of
 * width L_z/nslices (the analysis grid's GridZCellNo) and keeps it, in FP64,
 * per type pair [slice][t1*T+t2][9], per bond type [slice][bond_type][9] and
 * per bond-pair type [slice][bondpair_type][9]; bond_type[i] and
 * bondpair_type[i] give the type of every uploaded bond and bond pair
 * (CBond/CBondPair::GetType), nbondtypes/nbptypes their counts.  Bead 1 of a
 * pair is the reference's for pairs in different cells; inside one cell the
 * split between t1*T+t2 and t2*T+t1 can differ from the reference's (its
 * list order), so only their sum is comparable.  A degenerate bond pair
 * (|b1||b2| <= 1e-4) adds zero.  Single-box engines; call after the topology
 * upload, which turns the profile off again.  nslices = 0 turns it off. */
DPD_API int dpd_engine_set_slice_stress(dpd_engine* e, int32_t nslices, int32_t nbondtypes, const int32_t* bond_type,
                                        int32_t nbptypes, const int32_t* bondpair_type);
/* The slice stress profile of the latest sample step (synchronous); arrays
 * sized as above, any pointer may be NULL. */
DPD_API int dpd_engine_slice_stress(dpd_engine* e, double* pair, double* bond, double* bondpair);

/* CMonitor sample data beyond dpd_obs, computed on the device from the
 * current state when dpd_engine_monitor is called (so a sample needs no state
 * download):
 *   CalculateSingleBeadData     Monitor.cpp:790-1040  inertia tensor / N,
 *                               per-type MSD / (6 dt t N_type) from the initial
 *                               unPBC positions (at t = 0: / N_type)
 *   CalculateSinglePolymerData  Monitor.cpp:708-788   mean end-to-end distance
 *                               per polymer type (head - tail, minimum image)
 *   CalculateSingleBondData     Monitor.cpp:1052-1174 mean bond length per bond
 *                               type, global mean and mean square
 *   CalculateSingleBondPairData Monitor.cpp:1176-1273 per bond-pair type: P2,
 *                               first and second bond length, phi - phi0, its
 *                               square, and the ratio <dphi^2>/<dphi>^2
 * dpd_engine_set_monitor gives the bond and bond-pair types of the uploaded
 * topology, the polymers (head and tail bead ids, type) and the initial
 * unPBC positions (3 per bead in upload order; NULL = the current ones).
 * Call it after the topology upload; an upload of beads or topology clears it.
 * Single-box engines. */
typedef struct dpd_monitor {
    int64_t step;             /* m_SimTime of the state                             */
    int64_t n;
    double  inertia[9];       /* m_totalInertia / N, row-major (symmetric)          */
    int64_t bonds;
    double  mean_bond_length; /* over all bonds                                     */
    double  mean_sq_bond_length;
} dpd_monitor;
DPD_API int dpd_engine_set_monitor(dpd_engine* e, int32_t nbondtypes, const int32_t* bond_type, int32_t nbptypes,
                                   const int32_t* bondpair_type, int64_t npoly, const int64_t* poly_head_id,
                                   const int64_t* poly_tail_id, const int32_t* poly_type, int32_t npolytypes,
                                   const double* initial_unpbc3);
/* Synchronous.  msd[ntypes], bond_length[nbondtypes], end_to_end[npolytypes],
 * bondpair[6 * nbptypes] (P2, first length, second length, dphi, dphi^2,
 * dphi ratio); any array may be NULL. */
DPD_API int dpd_engine_monitor(dpd_engine* e, dpd_monitor* out, double* msd, double* bond_length,
                               double* end_to_end, double* bondpair);

/* Restart state in the reference's text format (CRestartState::Serialize,
 * RestartState.cpp:100-163), written from the device state without a round
 * trip through bead objects.  The layout is registered once: order[k] is the
 * upload index of the k-th bead of the file (the reference writes polymer by
 * polymer, beads in polymer order), poly_id[k] / poly_type[k] its polymer's
 * id and type, radius_by_type the bead radii.  An upload clears it.  The
 * file holds the constraint flags, then per bead: polymer id, polymer type,
 * bead id, bead type, radius, x[3], unPBC[3], v[3], F[3], with the stream's
 * default 6-significant-digit formatting; coordinates within 0.001 of a box
 * face are written as 0.001 and one outside the box is an error
 * (CheckBeadWithinBox, RestartState.cpp:488-530).  Synchronous. */
DPD_API int dpd_engine_set_restart_layout(dpd_engine* e, int64_t n, const int64_t* order, const int64_t* poly_id,
                                          const int32_t* poly_type, const double* radius_by_type);
DPD_API int dpd_engine_write_restart(dpd_engine* e, const char* path, int32_t wall, int32_t gravity, int32_t shear);

/* Writes a Paraview snapshot of n beads given in file order, from host
 * arrays (no device work): the file CCurrentState::Serialize writes with
 * CParaviewFormat (CurrentState.cpp:163-244, ParaviewFormat.cpp:72-112) --
 * header, one "x y z" line per bead at 6 significant digits, the vertex
 * list, one display id per bead.  Returns DPD_E_ARG when the file cannot be
 * written. */
DPD_API int dpd_write_paraview(const char* path, int64_t n, const double* x3, const int32_t* display_id);

/* The engine's current state as that Paraview snapshot, replacing
 * CCurrentState::Serialize for the Paraview format (from one position
 * download, no bead objects).  Beads are written by CNT cell in index order,
 * as CSimBox::GetAllBeadsInCNTCells lists them (SimBox.cpp:5883-5895); inside
 * a cell the reference follows its cell-list history and the engine the
 * upload order, so the files agree cell by cell.  type_visible (one byte per
 * bead type, NULL = all visible) leaves out invisible types as
 * CCurrentState does; display_id (per bead in upload order, NULL = the bead
 * type, the reference's default display map, Monitor.cpp:277) sets the
 * ptype column.  Single-box engines. */
DPD_API int dpd_engine_write_paraview(dpd_engine* e, const char* path, const uint8_t* type_visible,
                                      const int32_t* display_id);

/* Queues all further work on the caller's CUDA stream (a cudaStream_t passed
 * as a plain pointer; NULL returns to the engine's own stream).  The stream
 * must belong to the engine's device and outlive its use. */
DPD_API int dpd_engine_set_stream(dpd_engine* e, void* cuda_stream);

/* on = 1 starts recording CUDA events around every kernel the engine queues
 * (clearing earlier records); on = 0 stops.  Timing only, no extra sync. */
DPD_API int dpd_engine_profile(dpd_engine* e, int32_t on);

/* Waits for queued work and returns, per DPD_KERNEL_* id, the summed kernel
 * time in ms and the number of timed launches since profiling was switched on.
 * Both arrays hold DPD_NUM_KERNELS entries; either may be NULL. */
DPD_API int dpd_engine_profile_read(dpd_engine* e, double* total_ms, int64_t* launches);

/* Kernel launches the engine has queued since creation. */
DPD_API int64_t dpd_engine_launch_count(const dpd_engine* e);

DPD_API const char* dpd_engine_last_error(const dpd_engine* e);
DPD_API void dpd_engine_destroy(dpd_engine* e);

/* ---- Replica batches ---------------------------------------------------
 * A batch advances many independent boxes (replicas of different size, a_ij
 * and seed) with the same kernel launches: the boxes are packed into one
 * cell-sorted state and a box table, so a step costs one set of launches for
 * all of them.  The reference runs one box per process; each box of a batch
 * evolves exactly as the same box in its own engine.  dt, lambda, kT,
 * ntypes, precision and device come from `shared` (its box fields are
 * ignored).  Bonds are not supported in batches.  All dpd_engine_* calls
 * apply to a batch; positions in and out are box-local and dpd_engine_cells
 * reports box-local cell indices. */
DPD_API int dpd_batch_create(const dpd_params* shared, int32_t nboxes, const dpd_box* boxes, dpd_engine** out);

/* Beads of all boxes at once; box[i] is the box of bead i (ids may repeat
 * across boxes: each box has its own noise stream). */
DPD_API int dpd_batch_upload_beads(dpd_engine* e, int64_t n, const int32_t* box, const int64_t* id,
                                   const int32_t* type, const uint8_t* movable, const double* x3,
                                   const double* unpbc3, const double* v3, const double* f3);

/* Single-bead sums of one box (the virial from its latest sample step). */
DPD_API int dpd_batch_observables(dpd_engine* e, int32_t box, dpd_obs* out);

/* ---- z-slab decomposition, slab resident on the device ------------------
 * Replaces the reference's spatial decomposition over processors (the mps*
 * boxes: SimBox.cpp:481-567, mpsSimBox.cpp:796-860, CNTCell.cpp:3598
 * UpdateForceP) for a box split into slabs of whole CNT cell layers along z,
 * one per rank.  Each rank's engine is created for its local box: the global
 * box's nx, ny and widths, and z1 - z0 + 2*ghost layers (its own layers
 * [z0, z1) of the global nz_global, plus ghost layers on either side), with
 * positions in the local frame (global z minus (z0 - ghost) * wz, wrapped
 * into the global box; unPBC z minus the same).  The owned beads are
 * uploaded with dpd_engine_upload_beads; then every exchange is
 *   dpd_engine_slab_pack -> the caller sends send_below to the rank below and
 *   send_above to the rank above and receives the matching buffers
 *   (ncclSend/ncclRecv or any transport; the buffers are device memory) ->
 *   dpd_engine_slab_unpack,
 * once after setup (the first ghosts) and once after every
 * dpd_engine_step(e, t, 1).  The pair noise is keyed on bead ids and the step,
 * so every owned bead sees exactly the forces it sees in the whole box and no
 * force travels back.  In upload order the local beads are the owned ones
 * first (dpd_engine_download returns them in the first n_owned rows), then
 * the ghosts.  Calls that describe a whole box (bead uploads and builders,
 * topology uploads, observables, renormalisation, the slice profile, the
 * monitor, restart and snapshot layouts) return DPD_E_STATE on a slab. */

/* Turns an engine holding its slab's owned beads (the first n_owned of the
 * upload; all of them normally) into a slab, and takes the WHOLE box's
 * topology (bead ids 1..id_max): each exchange keeps the bonds and bond pairs
 * whose beads are all in the local box, on the device.  Needs ghost >= 1,
 * z1 - z0 >= 2*ghost and (z1 - z0) + 2*ghost <= nz_global.  Captured graphs
 * are off for a slab (its bead count changes every step). */
DPD_API int dpd_engine_slab_setup(dpd_engine* e, int32_t nz_global, int32_t z0, int32_t z1, int32_t ghost,
                                  int64_t n_owned, int64_t id_max, int64_t nb, const int64_t* bond_head_id,
                                  const int64_t* bond_tail_id, const double* k2, const double* l0, int64_t na,
                                  const int64_t* first_bond, const int64_t* second_bond, const double* k3,
                                  const double* phi0);

/* Packs the beads to send (asynchronous, on the engine's stream): migrants
 * (owned beads that left [z0, z1)) and the next step's ghosts (owned beads
 * within ghost layers of a face), as records of 16 doubles (id, type,
 * movable, kind, x[3], unPBC[3], v[3], F[3]; global frame) after a header
 * record (beads, of them migrants first, overflow flag).  Each buffer holds
 * (capacity + 1) * 16 doubles, 16-byte aligned, device memory. */
DPD_API int dpd_engine_slab_pack(dpd_engine* e, double* send_below, double* send_above, int64_t capacity);

/* Forms the next local box from this rank's staying beads and the two
 * received buffers (device memory; recv_below came from the rank below) and
 * uploads it on the device (no host copy of bead data; the call waits once
 * for the sizes).  Returns the owned and local bead counts.  DPD_E_LIMIT when
 * either side's beads overflowed a buffer, DPD_E_STATUS when the step before
 * set a fatal status bit (the state is then left as the step made it). */
DPD_API int dpd_engine_slab_unpack(dpd_engine* e, const double* recv_below, const double* recv_above,
                                   int64_t* n_owned, int64_t* n_local);

/* The current owned and local bead counts. */
DPD_API int dpd_engine_slab_counts(dpd_engine* e, int64_t* n_owned, int64_t* n_local);

/* Single-bead sums over this slab's owned beads, taken after a step and
 * before its exchange (synchronous): n (owned beads), sum_v, sum_v2, sum_x,
 * ang_mom (local frame), and the virial when the step was a sample step of
 * the full-shell pair scheme (has_virial; each bead of a pair holds half of
 * its virial there, so the ranks' sums count every pair once; bonds and bond
 * pairs count at the one bead that holds them).  kT and pressure are left 0:
 * the caller sums n, sum_v, sum_v2 and virial over the ranks (the FP64
 * all-reduce of CMonitor::CalculateSingleBeadData's terms) and forms
 * kT = sum_v2 / (3 n) and P = (sum_v2 + trace virial) / (3 V) of the whole box. */
DPD_API int dpd_engine_slab_observables(dpd_engine* e, dpd_obs* out);

/* ---- Pair forces without any allocation ---------------------------------
 * This entry point has no counterpart in the reference.  It is for callers
 * that may not allocate device memory at the moment they need forces: a host
 * program whose memory pool owns the whole GPU, a real-time loop where
 * cudaMalloc would stall the device, or a plug-in whose host forbids
 * library-side allocations.  Such a caller owns its bead and force buffers
 * but cannot give the engine the cell-list scratch it would otherwise
 * cudaMalloc (dpd_engine_create/upload).
 *
 * It computes the DPD pair forces of CCNTCell::UpdateForce (conservative,
 * dissipative and random; FP32 arithmetic, the engine's pair kernel) for
 * beads at positions x3 with the velocities v3 the forces should see (the
 * intermediate v~ of the step), types and noise ids, at timestep `step` (which
 * keys the pair noise), and writes them as FP64 to f3 in the caller's bead
 * order.  x3, v3, f3 (n*3 doubles, xyz interleaved), type and id (n int32)
 * are DEVICE pointers.  params->precision is ignored; params->device selects
 * the GPU (-1: current; the caller's current device is restored before the
 * call returns).  The work is queued on cuda_stream (NULL: the legacy
 * default stream) and the call is synchronous: it waits for that stream
 * (cudaStreamSynchronize) before it returns, to read its status word.
 *
 * Scratch: one fixed file-scope device array of about 4.5 MB, held by every
 * GPU that loads the library until the process exits.  Limits:
 * n <= DPD_NOALLOC_MAX_BEADS and nx*ny*nz <= DPD_NOALLOC_MAX_CELLS, otherwise
 * DPD_E_LIMIT with nothing launched.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and keeps it for the life of
 * the process; make that first call before any stream capture, and do not
 * reset the device's context (cudaDeviceReset) between calls.  All calls
 * share the one array and each call clears the parts that must start at
 * zero, so calls that overlap on the GPU (other threads or streams on the
 * same device) race and must be serialised by the caller.  Returns DPD_E_BOX
 * if a position lies outside the box (forces are then not meaningful),
 * DPD_E_ARG for bad arguments, including a bead type outside 0..ntypes-1
 * (found on the device; forces then not meaningful), DPD_E_CUDA on a CUDA
 * error.  No cudaMalloc, cudaFree or other allocating routine is called. */
#define DPD_NOALLOC_MAX_BEADS   65536
#define DPD_NOALLOC_MAX_CELLS   32768
DPD_API int dpd_pair_forces_noalloc(const dpd_params* params, int64_t step, int64_t n,
                                    const double* x3, const double* v3, const int32_t* type,
                                    const int32_t* id, double* f3, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* DPD_ENGINE_H */
