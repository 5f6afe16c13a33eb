// Host-side launch wrappers of the device kernels (build.cu, step_*.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"

namespace godar {

// Whether step kernels may be launched with programmatic dependent launch
// (GODAR_PDL=0: never).  Memory order is that of the stream either way,
// since every step kernel first waits for the kernel before it.
bool step_pdl();

// Launches a step kernel (one that starts with step_kernel_entry) on st,
// with programmatic dependent launch if pdl.
template <typename... Params, typename... Args>
inline void launch_step(bool pdl, void (*kern)(Params...), int grid, int block, cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t c = {};
    c.gridDim = dim3((unsigned)grid);
    c.blockDim = dim3((unsigned)block);
    c.dynamicSmemBytes = 0;
    c.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    c.attrs = at;
    c.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&c, kern, args...);
}

void scan_excl(const int *in, int *out, int n, int *scratch, cudaStream_t st);
void radix_sort(uint32_t *keys, int *vals, uint32_t *keys_alt, int *vals_alt, int n, int bits,
                int *counts, int *scratch, cudaStream_t st);
void launch_cell_keys(const Views &V, int cur, uint32_t *keys, int *vals, cudaStream_t st);
void launch_permute(const Views &V, int cur, const int *vals, const int *repack, int *old_slot, cudaStream_t st);
void launch_cell_ranges(const uint32_t *keys, int n, int *cstart, int *cend, cudaStream_t st);
void launch_nbr_count(const Views &V, int side, const int *cstart, const int *cend, int *cnt, cudaStream_t st);
void launch_nbr_fill(const Views &V, int side, const int *cstart, const int *cend, const int *row_off2,
                     int2 *ent2, double *dist2, int *nlo2, int up_by_id, cudaStream_t st);
void launch_nbr_link(const Views &V, const int *row_off2, const int *nlo2, int2 *ent2, cudaStream_t st);
void launch_split_rows(int N, const int *row_off2, const int *nlo2, const int2 *ent2, const int *lo_off,
                       const int *up_off, int2 *ent_lo, int2 *ent_up, cudaStream_t st);
void launch_row_lengths(int N, const int *row_off2, const int *nlo2, int *nup, cudaStream_t st);
void launch_migrate(const Views &V, int fp64, int side_new, const int *old_slot, const int *old_up_off,
                    const int2 *old_ent_up, const int *old_id, const void *old_hist, const int *up_off2,
                    const int2 *ent_up2, void *hist2, int *bidx2, cudaStream_t st);
void launch_copy_ids(const Views &V, int from, cudaStream_t st);

// The FP64 time step: (b) a screen of every owner entry (distance,
// candidate test, the entries that need no pair physics) and the pair
// physics once per work-list entry, writing pair records and flags; the
// ordered sums of every floe's records and its ridging events, into
// FP64_FLOE_SUMS doubles per floe; (c)-(e) walls, forcing and the FP64
// update (which also clears the work list).
constexpr int FP64_PAIR_REC_BYTES = 160;
constexpr int FP64_FLOE_SUMS = 18;
void launch_pairs_fp64_screen(const Views &V, int cur, int diag, int n, const int *plist, const unsigned *erow,
                              unsigned char *pfl, FP64Lists L, void *rec, int block, int variant, cudaStream_t st);
void launch_pairs_fp64_work(const Views &V, int cur, int diag, int list, int E, unsigned char *pfl, FP64Lists L,
                            void *rec, int block, cudaStream_t st);
void launch_row_sums_fp64(const Views &V, int cur, int diag, const unsigned char *pfl, const void *rec,
                          const int *lo_n, const int *up_n, double *fs, int block, cudaStream_t st);
// At a rebuild: the pairs that can act on a step without diagnostics before
// the next one marked (listed[p]), every row reordered to hold them first
// (up_n / lo_n per floe), and the list of their owner-row positions for the
// screen (plist, pos[N] of them; pos: N + 1 ints; tmp: 2 E entries).
void launch_fp64_rows(const Views &V, int side, int E, const unsigned *erow, unsigned char *listed, int *up_n,
                      int *lo_n, int2 *tmp, int *pos, int *scan_scratch, int *plist, cudaStream_t st);
void launch_floes_fp64(const Views &V, int cur, int diag, int sic, const double *fs, int *nwork, int block,
                       cudaStream_t st);
// Mixed precision: (b) one lane per pair with warp-segmented sums, (b') the
// partners' shares gathered the same way, (c)-(e) one thread per floe.
struct MixedBufs {
    unsigned char *pfl, *lfl;   // flags of the owner entries and of their mirror partner entries
    int *lo_of;                 // partner-row index of every owner entry
    float4 *rec;                // [2P] pair records: force/moments, shelter factors
    float2 *rx;                 // [P] ridging excesses of both floes
    float4 *pdg;                // [2P] diagnostic sums of the pair (diagnostic steps)
    float4 *brec, *bdg;         // [2NB], [4NB] bond records (per floe, slot order), diagnostic sums
    int *bfo;                   // [N+1] first bond record of every slot
    const BondGeom32 *bst;      // [NB] FP32 static bond records (working order)
    BondDyn *wdyn;              // [NB] dynamic bond records (working order)
    const int *winv;            // [NB] working index of every bond of the table
    const unsigned char *bfl_rd;   // [NB] live-bond flags at the start of the step
    unsigned char *bfl_wr;         // [NB] ... at its end (the other side)
    int4 *bsp;                  // [NB] slots of the bond's two floes, positions of their records (working order)
    int *blo_start, *blo_end;   // [N] by global id: range of the floe's partner bonds in blo_idx
    int *blo_idx;               // [NB] bond indices ordered by the higher id
    int *work, *nwork;          // [P] owner entries for the full pair computation, and their count
    int2 *work_st;              // [P] their row and partner slots (not on diagnostic steps)
    float4 *fsum;               // [2N] per floe: fcx fcy mc fbx | fby mb shelter(air) shelter(water)
    float *frex;                // [N] per floe: ridging excess
    float4 *fdg;                // [2N] per floe, diagnostic steps: tac pc tab pb | sxx syy sxy syx
    unsigned *dsp;              // [4] displacement bound of the contact-list screening: per side,
                                // the largest squared step of any floe (FP32 bits, rounded up),
                                // then per side the cumulative bound D (FP32 bits); zero at a rebuild
};
void launch_fill_erow(const int *off, int N, unsigned *erow, cudaStream_t st);
void launch_pack_snap(const Views &V, int side, cudaStream_t st);
void launch_mixed_rows_init(int P, const int2 *ent_lo, const void *hist, int *lo_of, unsigned char *pfl,
                            unsigned char *lfl, cudaStream_t st);
void launch_bond_slots(const Views &V, int side, int *slot_of, int4 *bsp, uint32_t *pkey, int *pval,
                       cudaStream_t st);
void launch_bond_work(const Views &V, int side, int nb, int *cnt, int *wfo, int *scan_scratch, int *perm,
                      const BondStat *in, const BondDyn *dyn, const int4 *bsp, BondGeom32 *wst, BondDyn *wdyn,
                      int4 *wsp, int *winv, unsigned char *wflag, cudaStream_t st);
void launch_bond_work_scatter(const int *perm, int nb, const BondDyn *wdyn, BondDyn *dyn, cudaStream_t st);
void launch_bond_positions(const Views &V, int side, const int *blo_start, const int *blo_end, const int *blo_idx,
                           int *cnt, int *bfo, int *scan_scratch, int4 *bsp, cudaStream_t st);
void launch_pairs_screen(const Views &V, int cur, int diag, int P, int2 *eb, const int2 *stl,
                         MixedBufs B, int block, int variant, cudaStream_t st);
void launch_contact_list(const Views &V, int side, int P, const unsigned *erow, const unsigned char *pfl, int *mark,
                         int *pos, int *scan_scratch, int2 *eb, int2 *stl, cudaStream_t st);
void launch_pairs_work(const Views &V, int cur, int diag, int P, const unsigned *erow_up, MixedBufs B, int block,
                       cudaStream_t st);
void launch_floe_sums(const Views &V, int diag, MixedBufs B, int block, cudaStream_t st);
void launch_bonds_mixed(const Views &V, int cur, int diag, int NB, MixedBufs B, int block, int variant,
                        unsigned test_spins, cudaStream_t st);
void launch_floes_mixed(const Views &V, int cur, int diag, int sic, int walls, MixedBufs B, int block,
                        cudaStream_t st);

// Checkpoints: pair histories out and back in.
void launch_hist_list(const Views &V, int cur, int off, int n, int fp64, int hs, int *count, int *pi, int *pj,
                      double *h4, int cap, cudaStream_t st);
void launch_hist_inject(const Views &V, int cur, int off, int nh, const int *pi, const int *pj, const double *h4,
                        int *slot_of, int fp64, int hs, unsigned char *pfl, cudaStream_t st);

// Output helpers.  Field codes GODAR_F_*; GATHER_DTB1 .. + 3: the wall
// histories deltat_bc1, deltat_bc2, theta_bc1, theta_bc2.
constexpr int GATHER_DTB1 = 100;
void launch_gather_field(const Views &V, int cur, int inst, int off, int n, int field, double *out, cudaStream_t st);
// Per instance: momentum x, y, kinetic energy, largest speed (4 doubles).
void launch_instance_summary(const Views &V, int cur, double *out, cudaStream_t st);
void launch_list_pairs(const Views &V, int cur, int inst, int off, int n, int which, int *pi, int *pj,
                       double *val, int cap, int *count, cudaStream_t st);

// Batch relayout (membership changes).
void launch_gather_floes(const Views &Vo, int so, const Views &Vn, int sn, const int *repack, int n, cudaStream_t st);
void launch_rebase_bond_off(const int *old_bond_off, int *new_bond_off, const int *inst, const int *old_slot_base,
                            const int *new_slot_base, const int *old_bbase, const int *new_bbase, int n,
                            cudaStream_t st);
void launch_gather_bonds(const int *old_hi, const BondStat *old_st, const BondDyn *old_dy, int *new_hi,
                         BondStat *new_st, BondDyn *new_dy, const int *bmap, int nb, cudaStream_t st);
void launch_set_int(int *p, int v, cudaStream_t st);

// Bond creation at admission (bonds_init.cu): cell list over the admitted
// floes [s0, s0 + n) on side `side`, per-floe bond counts and their scan;
// per-field totals; the bond table's entries of the fresh fields.
void launch_bond_init_count(const Views &V, int side, int s0, int n, const BondRule *rule, uint32_t *keys,
                            int *vals, uint32_t *keys_alt, int *vals_alt, int key_bits, int *rs_counts,
                            int *scan_scratch, int *cstart, int *cend, int *cnt, int *scan, cudaStream_t st);
void launch_bond_init_totals(const int *scan, const int *first, const int *last, int m, int *tot, cudaStream_t st);
void launch_bond_init_fill(const Views &V, int side, int s0, int n, const BondRule *rule, const int *cstart,
                           const int *cend, const int *vals, const int *scan, int *bond_off, int *bond_hi,
                           BondStat *bstat, BondDyn *bdyn, cudaStream_t st);

}  // namespace godar
