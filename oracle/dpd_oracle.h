/* dpd_oracle.h -- CPU restatement of Osprey-DPD's per-timestep DPD loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA engine is compared
 * against; the engine never links, loads or calls it.
 *
 * It restates, in plain C and in the reference's own operation order:
 *   CSimBox::Evolve                 SimBox.cpp:977-1120
 *   CCNTCell::UpdatePos             CNTCell.cpp:1598-2262 (27-way migration, PBC wrap)
 *   CCNTCell::UpdateForce (DPD)     CNTCell.cpp:1103-1572
 *   CCNTCell::UpdateMom             CNTCell.cpp:2280-2310
 *   CCNTCell::Randf / lcg           CNTCell.cpp:2454-2465
 *   CBond::AddForce                 Bond.cpp:111-162
 *   CBondPair::AddForce             BondPair.cpp:138-286
 *   CSimBox::MakeCNTCells / MapCelltoIndex / AssignBeadstoCells
 *                                   SimBox.cpp:715-940
 *   CCNTCell::CheckBeadsinCell      CNTCell.cpp:2628-2700
 *   CMonitor::AddBeadStress / AddBondStress / AddBondPairStress / ZeroSliceStress
 *                                   Monitor.cpp:1900-2755 (slice stress profile)
 *
 * Two noise sources are provided:
 *   DPDO_NOISE_LCG    - the reference's single 64-bit LCG consumed once per
 *                       interacting pair in cell-list order.  With this source
 *                       the oracle reproduces the reference bit for bit
 *                       (checked against the reference binary, oracle/_ref).
 *   DPDO_NOISE_PHILOX - Philox2x32-10 keyed on (step, min id, max id): the
 *                       order-independent, pair-symmetric stream the CUDA
 *                       engine uses, so GPU and oracle trajectories can be
 *                       compared with the thermostat on.
 */
#ifndef DPD_ORACLE_H
#define DPD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { DPDO_NOISE_LCG = 0, DPDO_NOISE_PHILOX = 1 };

typedef struct dpdo_params {
    int32_t nx, ny, nz;          /* CNT cells per axis (Box nx ny nz)          */
    double wx, wy, wz;           /* CNT cell widths    (Box ... wx wy wz)      */
    double dt, lambda, kT;       /* Step, Lambda, Temp                         */
    int32_t ntypes;              /* bead types                                 */
    const double* a;             /* ntypes*ntypes conservative a_ij (row-major) */
    const double* gamma;         /* ntypes*ntypes dissipative gamma_ij          */
    uint64_t seed;               /* |RNGSeed| (CNTCell.cpp:134-137)            */
    int32_t noise;               /* DPDO_NOISE_*                               */
} dpdo_params;

typedef struct dpdo_sim dpdo_sim;

dpdo_sim* dpdo_create(const dpdo_params* p);
void dpdo_destroy(dpdo_sim* s);

/* Beads in the reference's bead-vector order (bead id order); this order
 * fixes the initial cell-list order exactly as AssignBeadstoCells does. */
int dpdo_set_beads(dpdo_sim* s, int64_t n, const int64_t* id, const int32_t* type,
                   const uint8_t* movable, const double* x3, const double* unpbc3,
                   const double* v3, const double* f3);

/* Bonds by bead id (head, tail); bond pairs by index into the bond list. */
int dpdo_set_topology(dpdo_sim* s, int64_t nb, const int64_t* head_id, const int64_t* tail_id,
                      const double* k2, const double* l0, int64_t na,
                      const int64_t* first_bond, const int64_t* second_bond,
                      const double* k3, const double* phi0);

/* Runs nsteps timesteps; first_step is the reference's m_SimTime of the first. */
int dpdo_step(dpdo_sim* s, int64_t first_step, int32_t nsteps);

/* State in set_beads order; any pointer may be NULL. */
int dpdo_get(const dpdo_sim* s, double* x3, double* unpbc3, double* v3, double* f3,
             double* stress9);

/* Cell index each bead's list belongs to (set_beads order). */
int dpdo_get_cells(const dpdo_sim* s, int32_t* cell);

/* Beads whose floor(x/w) cell differs from their list cell after the last step. */
int64_t dpdo_cell_errors(const dpdo_sim* s);

/* Interacting pairs (r < 1, r > 1e-9) found in the last force evaluation. */
int64_t dpdo_pair_count(const dpdo_sim* s);

/* Philox2x32-10 draw used for the pair noise: first output word. */
uint32_t dpdo_philox_pair(uint64_t seed, int64_t step, uint32_t id_lo, uint32_t id_hi);

/* Slice stress profile of CMonitor (Monitor.cpp:1900-2755, zeroed every
 * step as SimBox.cpp:999): nslices z slices of width L_z/nslices (the
 * analysis grid's GridZCellNo), pair part indexed [slice][type1*T+type2][9]
 * with bead 1 the reference's iterating bead, bond part [slice][bond type][9],
 * bond-pair part [slice][bondpair type][9].  nslices = 0 turns it off.  Call
 * after dpdo_set_topology. */
int dpdo_set_slice_stress(dpdo_sim* s, int32_t nslices, int32_t nbondtypes, const int32_t* bond_type,
                          int32_t nbptypes, const int32_t* bondpair_type);
int dpdo_get_slice_stress(const dpdo_sim* s, double* pair, double* bond, double* bondpair);
/* Contributions that fell outside the slices (a z at the box edge rounded up). */
int64_t dpdo_slice_errors(const dpdo_sim* s);

/* Time-step dependent constants after a ChangeTimeStepConstants (CNTCell.cpp:357). */
int dpdo_set_dt(dpdo_sim* s, double dt);
/* a_ij / gamma_ij update (CNTCell.cpp:434-456 sets both (i,j) and (j,i)). */
int dpdo_set_pair(dpdo_sim* s, int32_t ti, int32_t tj, double a, double gamma);
/* CSimBox::UpdateRenormalisedMom (SimBox.cpp:3177-3225): momenta rescaled to kT. */
int dpdo_renormalise_mom(dpdo_sim* s);

/* Random initial state of CRandomBuilder::Assemble (RandomBuilder.cpp:71-361,
 * no walls, 3-d): positions x3 and velocities v3 (3 per bead, bead order) for
 * n beads in a box of lengths L at temperature kT, from the reference's LCG
 * seeded with `seed` after `skip` draws; bonds (bead indices, polymer order)
 * shorten long bonds as the reference does.  The unPBC position equals x3.
 * Returns 0, or -1 - i when bead i falls outside the box. */
int dpdo_random_state(int64_t n, const double L[3], double kT, uint64_t seed, int64_t skip, int64_t nb,
                      const int64_t* bond_head, const int64_t* bond_tail, double* x3, double* v3);
/* CLamellaBuilder::Assemble restated (no walls, no polymerised bonds); see
 * dpd_oracle.c.  Returns 0, -1 bad arguments, -2 bilayer outside the box,
 * -3 lattice outside the box. */
int dpdo_lamella_state(int64_t n, const double L[3], double kT, uint64_t seed, int64_t skip, int64_t npoly,
                       const int64_t* poly_first, const int32_t* poly_type, int32_t lipid_type,
                       int32_t head_offset, int32_t tail_offset, int32_t normal, double centre_frac,
                       double thickness, int32_t linearise, double upper_fraction, int64_t nb,
                       const int64_t* bond_head, const int64_t* bond_tail, double* x3, double* v3);

#ifdef __cplusplus
}
#endif

#endif
