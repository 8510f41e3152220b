// A FoF plan: run parameters, device workspace and the last run's outputs.
#pragma once

#include <vector>

#include "cmh_internal.cuh"
#include "fof_kernels.cuh"

struct cmh_plan {
  virtual ~cmh_plan() = default;
};

namespace cmh {

struct Plan : public cmh_plan {
  int device = 0;
  cmh_fof_params params{};
  std::vector<double> ltab_host;
  int pos_dtype = CMH_FLOAT32;
  bool fp32 = true;
  uint32_t dense_min = 16;  // top cells with more occupied fine cells get a map

  Geom geom{};
  uint64_t n_top = 0;
  int key_bits = 0;
  cmh_stats stats{};
  int64_t out_nhalos = 0;

  uint32_t *h_scal = nullptr;  // pinned host copy of the device scalars
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t stage_ev[7] = {};  // boundaries between the eight stages

  // workspace
  DevBuf scal, ctr, scan_tmp, sort_tmp, ltab_dev;
  DevBuf b_keep, b_nimg, b_keep_scan, b_img_scan;
  DevBuf b_keys, b_keys_alt, b_vals, b_vals_alt, b_ppos, b_spos, b_run_of;
  DevBuf b_run_start, b_run_g, b_top_first, b_top_end, b_top_slot, b_rtmp1, b_rtmp2, b_maps;
  DevBuf b_parent, b_count, b_head, b_cand_of_root, b_cand_root, b_sums, b_warn;
  DevBuf b_own, b_own_scan, b_okeys, b_ovals, b_okeys_alt, b_ovals_alt;
  DevBuf b_props, b_head_out, b_cat_of_cand, b_member, b_member_proc, b_member_pos;
  DevBuf in_pos, in_vel;  // device copies of host-resident particles
  DevBuf b_dense_range;   // first/end fine cell of each dense top cell

  Plan(const cmh_fof_params &p, int pos_dtype, int device);
  ~Plan() override;
  void set_params(const cmh_fof_params &p);
  void setup_geometry(int64_t n_in);
  void run(const cmh_particles &parts, bool want_member, cudaStream_t s);
  template <class PT, class VT>
  void run_typed(const cmh_particles &parts, bool want_member, cudaStream_t s);
};

}  // namespace cmh
