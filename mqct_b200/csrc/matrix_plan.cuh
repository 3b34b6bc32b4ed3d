// matrix_plan.cuh -- state of one matrix-build plan (uploaded system, grids,
// GEMM row order) shared by the FP64 and tcgen05 contraction paths.
#pragma once
#include <memory>
#include <vector>

#include "common.cuh"

namespace mqct {

// Surrogate bridge (surrogate.cu).
int surrogate_predict_on(void* sur, const float* X, int64_t n, double* v_out, cudaStream_t st);
void surrogate_feature_map(const void* sur, int* sys_type, double* r_c, double* r_s);

// Per-plan state of the tcgen05 path (contract_tc.cu).
struct TcInfo {
  int n_chunks = 0, chunks_per_split = 1, npad = 0, nbmax = 0;
  int n_parts = 1, part_c0[8] = {}, part_nc[8] = {};  // column parts of the radial axis
  int nbuf = 2;                                        // B / basis-slice buffers
  int slices_per_drain = 1;                            // alpha points per FP64 drain
  bool alpha_uniform = true;                           // all alpha weights equal
  int pe_warps = 8;                                    // epilogue warps of the last launch
  int pe_force = 0;                                    // 8 or 16 (tuned or set), 0: by rule
  float pe_tune_ms[2] = {0.f, 0.f};                    // contraction ms with 8 and 16
  uint32_t b_stage = 0, psi_stage = 0;                 // bytes of one such buffer
  int n_blocks = 0, n_sm = 148;
  size_t smem = 0;
  DevBuf<int> blk_row0, blk_n, blk_m;
  DevBuf<int64_t> blk_img_off;
  DevBuf<double> walpha;
  DevBuf<int> wexp;  // F16x3: power-of-two exponent of each W column
};

struct MatrixPlan {
  // problem
  int sys_type = 0, precision = 0;
  int64_t P = 0;
  int nR = 0, n_states = 0;
  int G2 = 0;        // 2-D grid points (beta x gamma) or beta points (type 1)
  int n_gamma = 1;
  int n_alpha = 0;   // explicit alpha grid points (0: analytic 2*pi)
  int ldv = 1;
  int ir1 = 0, ir2 = 0;
  double cut = 0.0;
  int pes_kind = 0, pes_n_terms = 0, pes_n_sites1 = 0, pes_n_sites2 = 0;
  std::vector<double> Rh, h_beta, h_gamma, h_wt, h_alpha, h_walpha;
  // SYS_TYPE 3 runs as SYS_TYPE 4 on the parity-adapted top vectors held here
  std::vector<double> sym_top_vec;
  mqct_sys_t sym_top_sys{};
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};

  // GEMM rows: pairs grouped by m-block, each block padded to a multiple of 128
  int n_rows = 0, n_tiles = 0, n_basis_rows = 0;
  std::vector<int> h_rowa, h_rowb, h_tile_block;
  std::vector<int> h_block_row0, h_block_n, h_block_m;  // m-blocks of the basis rows
  DevBuf<int> d_rowa, d_rowb, d_rowm, d_k2r, d_tile_block;
  DevBuf<int> d_row_state, d_st_chan, d_st_m, d_ch_j;
  DevBuf<double> d_vec, d_beta, d_gamma, d_wt, d_alpha, d_walpha, d_R;
  DevBuf<double> d_pes_p, d_pes_s1, d_pes_s2, d_pes_table;
  // SYS_TYPE 0: second rotor, Clebsch-Gordan table, the extra grid axes
  DevBuf<int> d_ch_j2;
  DevBuf<double> d_vec2, d_cg, d_beta2, d_alpha2, d_gamma2;
  int cg_ld = 1, t0_nbb = 1, t0_naa = 1, t0_ngg = 1;
  // type 4: rotor d-function and gamma-phase tables (rebuilt by every execute)
  DevBuf<double> d_dtab;
  DevBuf<double2> d_phase;
  int jmax_basis = 0;
  // learned PES (surrogate.cu): features, network values, per-R residual ratios
  void* sur = nullptr;
  double sur_rel = 0.0, sur_abs = 1.0;
  int sur_check = 1;
  DevBuf<float> d_sur_x;
  DevBuf<double> d_sur_v;
  DevBuf<unsigned> d_sur_ratio;

  // work
  DevBuf<double2> d_psi;  // basis rows x G2, FP64
  DevBuf<double> d_W;     // G2 x ldw, FP64
  int ldw = 0;
  DevBuf<double> d_acc;   // FP64 form: n_rows x nR
  DevBuf<double> d_spl_fin;   // grid-only coefficients of the fused spline fit
  DevBuf<double> d_col_scale; // F16x3: exact per-column rescaling of the contraction

  // tcgen05 split-precision paths (contract_tc.cu)
  int tc_splits = 1, tc_ldp = 0, tc_npad = 0, tc_nchunk = 0;
  DevBuf<double> d_part;                // tc_splits x n_rows x tc_ldp FP64 sums
  DevBuf<unsigned short> d_bimg;        // pre-swizzled B (W) images, hi/lo planes
  DevBuf<float2> d_psi32;               // basis in FP32, chunk-major per row
  DevBuf<int> d_status;
  std::unique_ptr<TcInfo> tc;
  int tc_init();
  int tc_execute();
  int tc_check_status();
  int error_report(const double* d_mat, mqct_err_report_t* err);

  int init(const mqct_sys_t* sys, const int32_t* ind_mat, int64_t P, const double* R, int32_t nR,
           const mqct_grid_t* grid, const mqct_pes_t* pes, int32_t prec, double mij_cut,
           double rc1, double rc2);
  int refresh_inputs(const mqct_sys_t* sys, const double* R, const mqct_pes_t* pes);
  int run_basis_and_pes();
  int run_surrogate_pes(const struct PesDev& pd, const struct Type0Dev& t0);
  int execute(double* d_mat, double* d_y2, int32_t* d_skipped);
  double flops() const;
  ~MatrixPlan();
};

}  // namespace mqct
