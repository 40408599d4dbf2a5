// Device-resident plan of one sparsity pattern and the value layout of one instance.
//
// Value layout ("blob") of one instance, FP64, 256-byte aligned, instance-major:
//   [0, S)                 sparse slots: every filled-pattern entry that is not in the dense
//                          trailing block, in CSC order (so for columns c < t slot == CSC
//                          position, and L(:,c) is a contiguous run)
//   [dbase, dbase+ntp^2)   dense trailing block D = rows/cols [t, n), column-major with
//                          leading dimension ntp = round_up(n - t, 64); the padding is an
//                          identity block, so every dense kernel works on whole 64-tiles
// A plan with no dense block has t = n, ntp = 0.
#pragma once

#include <cstdint>

namespace glu {

constexpr int kDenseAlign = 64;     // ntp is a multiple of this
constexpr int kMaxPanel = 64;

// Geometry of one front's dense buffer: its offset in an instance's front area, its first entry
// in the pivot-perturbation flags (fhasl), leading dimension (= rows: padded pivots + padded rows
// below), columns (padded pivots + padded columns to the right), pivots and padded pivots.
struct FrontGeom {
  int64_t foff, h_off;
  int32_t ld, cols, w, wp;
};

struct PlanDev {
  // pattern
  uint32_t n, nnz, t, nt, ntp;
  int64_t S, dbase, blob;            // value slots per instance (blob is 32-aligned)
  // sparse phase (columns c < t)
  const uint32_t* cp;                // sym_c_ptr [n+1]
  const uint32_t* ri;                // sym_r_idx [nnz]
  const uint32_t* lp;                // l_col_ptr [n]
  const uint32_t* lsplit;            // [t] number of L(:,c) rows < t
  const int64_t* pair_ptr;           // [t+1] range of U(c,:) pairs of column c
  const int32_t* pair_j;             // [npairs] column j of U(c,j)
  const int32_t* pair_uslot;         // [npairs] slot of U(c,j)
  const int64_t* pair_moff;          // [npairs] offset of the row-position run in tmap
  const int32_t* tmap;               // [nmap] target slots of sparse targets
  const int32_t* scols;              // sparse columns in level order
  // sparse-to-dense contributions: hub columns (gathered panels, one DMMA GEMM) ...
  int32_t hubs_p;                    // hub count rounded up to 16 (GEMM K); 0 = no hub update
  int64_t ngl, ngu;
  const int32_t* gl_src;             // [ngl] slot of an L21 entry of a hub column
  const int32_t* gl_dst;             // [ngl] index in G_L (ntp x hubs_p, column-major)
  const int32_t* gu_src;             // [ngu] slot of a U12 entry of a hub column
  const int32_t* gu_dst;             // [ngu] index in G_U (hubs_p x ntp, column-major)
  // ... and every other column, pulled per tail column
  int64_t npull;
  const int64_t* pull_ptr;           // [nt+1]
  const uint32_t* pull_lb;           // [npull] entries [pull_lb, pull_le) of the CSC arrays: the
  const uint32_t* pull_le;           //   dense-block rows of L21(:,c), c with U(c, j) != 0
  const int32_t* pull_uslot;         // [npull] slot of U(c, j)
  const int64_t* pull_mend;          // [nt] or null: end of the entries of a column's own CTA
  const int32_t* pull_xcol;          // [npullx] column of each extra chunk of entries
  const int64_t* pull_xe;            // [2 npullx] the chunk's entries [xe[2k], xe[2k+1])
  int64_t npullx;
  // fronts (supernodal runs of sparse columns)
  const int32_t* fg_slot;            // gather / write-back: slot ...
  const int32_t* fg_idx;             // ... and index in the front buffer
  const int32_t* fc_slot;            // Schur complement: target slot ...
  const int32_t* fc_idx;             // ... and index in the front buffer
  const uint8_t* fhasl;              // pivot may be perturbed, per padded front pivot
  const int32_t* fs0;                // first column of every front
  const int32_t* fw;                 // width of every front
  int32_t fw_max;                    // widest front
  const int32_t* lfr;                // fronts in L-solve level order
  const int32_t* ufr;                // fronts in U-solve level order
  const FrontGeom* fgeom;            // [fronts]
  const int32_t* fg_aidx;            // gather / write-back index within an instance's front area
  const int32_t* fc_aidx;            // Schur-complement index within an instance's front area
  // dense phase
  const uint8_t* dhasl;              // [ntp] column of D has a non-empty L part (perturbation)
  // value ingest / export
  const int64_t* pos2slot;           // [nnz] filled-pattern position -> slot
  int64_t nnz_a;
  const int64_t* ing_slot;           // [nnz_a] slot of each original entry (-1 = dropped)
  const double* ing_scale;           // [nnz_a] or nullptr
  // rows of dense column j that the ingest writes: asm_row[asm_ptr[j] .. asm_ptr[j+1]), j < ntp
  // (the dense block is then assembled column by column instead of cleared beforehand)
  const int32_t* asm_ptr;            // [ntp+1] or nullptr
  const int32_t* asm_row;
  // dense slots that fronts add their Schur complements to: cleared by the load, kept (like the
  // ingested entries) by the assembly
  int64_t nasm_zero;
  const int32_t* asm_zero;
  // solve
  const uint32_t* col_perm;          // [n]
  const uint32_t* row_perm_inv;      // [n]
  const uint32_t* row_perm;          // [n]
  const double* col_scale_perm;      // [n] or nullptr
  const double* row_scale;           // [n] or nullptr
  const int32_t* lcols;              // sparse columns in L-solve level order
  const int32_t* ucols;              // sparse columns in U-solve level order
  const int64_t* bord_ptr;           // [nt+1] border entries U(r<t, j>=t) of tail column j
  const int32_t* bord_row;           // [nbord]
  const int32_t* bord_slot;          // [nbord]
  const int32_t* bord_ckcol;         // [nbordck] chunks of <= 1024 border entries: tail column
  const int64_t* bord_ck0;           //   and first entry
  int64_t nbordck;
  // original matrix pattern (gradient, residual): entry e is A(g_row[e], g_col[e])
  int64_t nnz_g;
  const uint32_t* g_row;             // [nnz_g]
  const uint32_t* g_col;             // [nnz_g]
  const int64_t* o_row_ptr;          // [n+1] entries of each row ...
  const int64_t* o_row_e;            // [nnz_g] ... (entry indices, row-major order)
  const int64_t* o_col_ptr;          // [n+1] entries of each column ...
  const int64_t* o_col_e;            // [nnz_g] ... (column-major order)
  // deterministic mode (see plan_host.h): per-target pair lists and the CSR mirror with slots
  const int64_t* det_q;              // pairs, grouped by target column
  const int32_t* det_c;              // their source columns
  const int64_t* det_tptr;           // [targets + 1]
  const uint32_t* rp;                // csr_r_ptr [n+1]
  const uint32_t* ci;                // csr_c_idx [nnz]
  const uint32_t* dp;                // csr_diag_ptr [n]
  const int32_t* csr_slot;           // [nnz] slot of each CSR entry (-1 inside the dense block)
};

}  // namespace glu
