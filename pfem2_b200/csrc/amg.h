// amg.h -- smoothed-aggregation multigrid for the pressure Poisson systems:
// the host-side hierarchy (built once at setup from the eliminated FP64
// matrix) in the layout the persistent solver kernel reads.
//
// The reference preconditions its pressure solve with Trilinos ML
// (TrilinosWrappers::PreconditionAMG, TurekBenchmarkCuda/TurekBenchmark.cc:
// 731-797). Here one V(1,1) cycle with damped Jacobi smoothing and
// smoothed-aggregation transfers is applied in its additive form
//   M_l^-1 = J_l + Pt_l M_{l+1}^-1 Pt_l^T,
//   J_l  = 2 w D^-1 - w^2 D^-1 A_l D^-1,  Pt_l = (I - w D^-1 A_l) P_l,
// which is algebraically the same V-cycle: the pre- and post-smoothing of a
// level are folded into J_l and into the post-smoothed prolongator Pt_l, so
// a level costs one sparse product each way and no extra synchronisation.
// Levels: 0 = the pressure rows; 1, 2 = aggregates of the level below built
// inside each solver tile; 3 = one aggregate per tile, solved exactly with
// a dense inverse.
#pragma once
#include <vector>

#include "ctx.h"

namespace pfem2 {

constexpr int kMgLevels = 4;

struct MgHost {
  int n[kMgLevels] = {0, 0, 0, 0};        // dofs per level over all systems
  std::vector<int> toff[kMgLevels];       // [l][ntiles+1] first level-l dof of each tile (l >= 1)
  std::vector<int> lsys[kMgLevels];       // [l][n_l] system of each level-l dof (l >= 1)
  std::vector<int> lk[3];                 // [1..2][n_l] index of that system among its block's systems
  // restrictions from level 0 (CSR over the rows of level l, global
  // level-0 columns): R0l = (Pt_0 ... Pt_{l-1})^T, l = 1, 2; R02 only
  // without the split restriction
  std::vector<int> r01_ptr, r01_col, r02_ptr, r02_col;
  std::vector<double> r01_val, r02_val;
  // split restriction (large systems): b2 = Pt_1^T b1 in a phase of its
  // own, CSR over the level-2 rows with global level-1 columns
  bool split = false;
  std::vector<int> q2_ptr, q2_col;
  std::vector<double> q2_val;
  // b3 = Pt_2^T b2 in two steps: every block adds up the contributions of
  // its own level-2 rows to the level-3 dofs they touch (CSR rows c3,
  // columns = own level-2 row - first own row, grouped per block by c3_blk,
  // c3_lk = the dof's system among the block's systems) and stores row r at
  // c3_pos[r]; the contributions of level-3 dof d are then the contiguous
  // range [g3_ptr[d], g3_ptr[d+1]) of that array, in block order
  std::vector<int> c3_blk, c3_ptr, c3_col, c3_lk, g3_ptr, c3_pos;
  std::vector<double> c3_val;
  // level-0 smoother J_0 on the SELL pattern of A
  std::vector<double> j0;
  // post-smoothed prolongator of level 0 on SELL slices; columns are the
  // indices into the owning block's level-1 list
  std::vector<int> p0_ptr, p0_len, p0_col;
  std::vector<double> p0_val;
  // per-block lists of the level-1 and level-2 dofs a block evaluates
  // (own dofs and the halo its prolongation reads): J rows (level 1:
  // global columns; level 2: the system's level-2 index), Pt rows with
  // columns into the block's next-level list
  std::vector<int> blk_s[3];              // [1..2][G+1] list offsets; [0] unused
  // (s_sys, s3_sys: index of the entry's system among the block's systems)
  std::vector<int> s_sys[3], s_jptr[3], s_jcol[3], s_pptr[3], s_pcol[3];
  std::vector<double> s_jval[3], s_pval[3];
  // per-block level-3 list: system, and where its column of the block's
  // transposed coarse-inverse rows starts (stride s3_estr)
  std::vector<int> blk_s3, s3_sys, s3_eoff, s3_estr, blk_e;
  std::vector<float> s3_E;
  std::vector<int> sys_D3, sys_off3;      // coarse size and first level-3 dof per system
  std::vector<int> sys_n2, sys_off2;      // level-2 size and first level-2 dof per system
  int s1max = 0, s2max = 0, s3max = 0, emax = 0, dmax = 1;
  int b2max = 0;                          // level-2 dofs of the local systems of a block
  // diagnostics
  std::vector<double> w;                  // smoother weight per system and level
};

// Builds the hierarchy of every pressure system. A, col, len: host copy of
// the eliminated FP64 pressure matrix in the context's SELL layout; tiles,
// st0: the pressure solve's tiles and first tile per system; bt0: first
// tile per block of the persistent grid; split: restrict to level 2 in a
// phase of its own (b2 = Pt_1^T b1) instead of through the composite R02;
// coarse_max: level-3 unknowns per system at most (groups of tiles share
// one), which bounds the dense inverse rows a block holds in shared memory.
pfem2_status mg_build(const Ctx& c, const std::vector<double>& A, const std::vector<int>& col,
                      const std::vector<int>& len, const std::vector<Tile>& tiles, const std::vector<int>& st0,
                      const std::vector<int>& bt0, bool split, int coarse_max, MgHost& out);

// In-place inverse of an SPD matrix (Cholesky, then L^-T L^-1); false if
// the matrix is not SPD.
bool spd_inverse(std::vector<double>& M, int n);

}  // namespace pfem2
