// A FoF plan: run parameters, device workspace, the captured graph of the
// last run shape and the last run's outputs.
#pragma once

#include <vector>

#include "cmh_internal.cuh"
#include "fof_kernels.cuh"

struct cmh_plan {
  virtual ~cmh_plan() = default;
};

namespace cmh {

// One domain of a run as the host describes it.
struct BoxSpec {
  cmh_fof_params params{};
  std::vector<double> ltab;
  const void *pos = nullptr;
  const void *vel = nullptr;
  bool vel_f64 = false;
  int64_t n = 0;
  int cell_factor = 0;  // 0: the params' value, or the autotuned one
};

struct Plan : public cmh_plan {
  int device = 0;
  cmh_fof_params params{};
  std::vector<double> ltab_host;
  int pos_dtype = CMH_FLOAT32;
  bool fp32 = true;
  bool use_graph = true;    // replay the captured run when its shape repeats
  uint32_t dense_min = 16;  // top cells with more occupied fine cells get a map
  double cell_scale = 1.0;  // autotuned scale of the default cell-size factor
  // bounds of the device loops that retry or wait (cmh_plan_set_limits)
  uint32_t union_cap = kUnionCap;  // retries of one union after a lost race
  uint32_t spin_cap = kSpinCap;    // polls of one sort tile state
  bool stall_sort = false;         // CMH_FAULT=lookback for this run

  // shape of the current run
  std::vector<BoxDev> boxes_host;
  int64_t n_total = 0;
  uint64_t n_top = 0, k3all = 1;
  int key_bits = 0, hs = 7, props = 0;
  bool varlink = false;             // some box has a variable linking length
  std::vector<double> ltab_all;     // their tables, back to back
  int64_t np_cap = 0, nd_cap = 0, nc_cap = 0;  // grown on overflow, never shrunk

  // results of the last run
  cmh_stats stats{};
  DevScal last{};
  std::vector<uint32_t> boxd_host;  // per box: 7 arrays of nbox (see k_box_totals)
  int64_t out_nhalos = 0;
  int32_t launches_per_run = 0;
  bool launches_per_run_graph_ok = false;

  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaStream_t bf_stream = nullptr;  // the dense top cells' kernel, beside the sparse one
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev_cleared = nullptr, ev_emitted = nullptr, ev_cleared2 = nullptr;
  cudaEvent_t stage_ev[7] = {};  // boundaries between the eight stages
  // the recorded graphs of the last two run shapes (two, so that runs that
  // alternate between the two host-input buffers both replay)
  cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};
  std::vector<unsigned char> graph_sig[2];
  int graph_next = 0;  // the slot the next recording replaces
  std::vector<unsigned char> uploaded_sig;  // shape whose box table is on the device
  cudaStream_t cap_stream = nullptr;  // the stream runs are recorded on
  // host-resident inputs: copied into one of two device buffers on a side
  // stream, positions first; a run waits for its positions before it starts
  // and for its velocities before the property sums (which are the first to
  // read them).  cmh_plan_prefetch stages the next run's inputs into the other
  // buffer while a run computes.  With one input buffer (input_buffers == 1)
  // the next run's copies go into the same buffer once the current run is
  // done with it: its positions after the current run's ingest (ev_pos_free)
  // and its velocities after its property sums (ev_vel_free).
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_side_start = nullptr, ev_pos[2] = {}, ev_vel[2] = {};
  cudaEvent_t ev_pos_free = nullptr, ev_vel_free = nullptr;
  cudaEvent_t ev_vel_ready = nullptr;  // the current run's (one of ev_vel)
  bool vel_wait = false;
  int input_buffers = 2;
  struct Staged {
    std::vector<cmh_particles> parts;  // the host inputs as given, one per box
    int buf;
    bool pending;  // one-buffer mode: not copied yet (waits for the run before)
  };
  std::vector<Staged> staged;  // inputs being copied ahead, oldest first (at most 2)
  int last_buf = 0;            // the buffer of the last run's inputs
  std::vector<cmh_particles> cur_host;  // host inputs of the run in progress
  bool overwritten = false;    // one-buffer mode: the next run's copies were queued
  // subsampling of the run's particles (FOF.c:205-284): rates, seed and the
  // particle IDs on the device (NULL: the input index is the key)
  bool sampling = false;
  double samp_in = 0.0, samp_out = 0.0;
  uint64_t samp_seed = 0;
  int samp_closed = 0;  // bit a: the domain includes its upper face on axis a
  const uint64_t *samp_ids = nullptr;

  // workspace
  DevBuf scal, ctr, scan_tmp, scan_tmp2, sort_tmp, ltab_dev, b_boxes, b_boxd;
  DevBuf b_keys, b_keys_alt, b_vals, b_vals_alt, b_ppos, b_spos, b_svl;
  DevBuf b_run_start, b_run_box, b_top_range, b_top_slot, b_rtmp1, b_rtmp2;
  DevBuf b_rows, b_dense_range, b_dense_big;
  DevBuf b_parent, b_count, b_head, b_cand_of_root, b_cand_root, b_sums, b_warn;
  DevBuf b_okeys, b_ovals, b_okeys_alt, b_ovals_alt;
  DevBuf b_props, b_head_out, b_cat_of_cand, b_member, b_member_proc, b_member_pos;
  DevBuf in_pos[2], in_vel[2];  // device copies of host-resident particles
  DevBuf b_samp;          // per input particle: 0, 1 (kept, in a halo), 2 (kept, outside)

  // every workspace buffer, for release and for the graph signature
  template <class F> void each_buf(F f) {
    DevBuf *all[] = {&scal, &ctr, &scan_tmp, &scan_tmp2, &sort_tmp, &ltab_dev, &b_boxes, &b_boxd,
                     &b_keys, &b_keys_alt, &b_vals, &b_vals_alt, &b_ppos, &b_spos, &b_svl,
                     &b_run_start, &b_run_box, &b_top_range, &b_top_slot,
                     &b_rtmp1, &b_rtmp2, &b_rows, &b_dense_range, &b_dense_big, &b_parent, &b_count,
                     &b_head, &b_cand_of_root, &b_cand_root, &b_sums, &b_warn,
                     &b_okeys, &b_ovals, &b_okeys_alt, &b_ovals_alt, &b_props,
                     &b_head_out, &b_cat_of_cand, &b_member, &b_member_proc, &b_member_pos,
                     &in_pos[0], &in_vel[0], &in_pos[1], &in_vel[1], &b_samp};
    for (DevBuf *b : all) f(*b);
  }
  void release_workspace();

  Plan(const cmh_fof_params &p, int pos_dtype, int device);
  ~Plan() override;
  void set_params(const cmh_fof_params &p);
  Geom make_geometry(const cmh_fof_params &p, const std::vector<double> &ltab, int64_t n_in,
                     int cell_factor) const;
  void prepare(const std::vector<BoxSpec> &specs, bool want_member);
  template <class PT>
  void issue(bool want_member, cudaStream_t s, bool timed);
  void read_back(cudaStream_t s, bool timed);
  void capture(bool want_member, cudaStream_t s, const std::vector<unsigned char> &sig);
  void run_batch(const std::vector<BoxSpec> &specs, bool want_member, cudaStream_t s);
  cmh_tuning autotune(const std::vector<BoxSpec> &specs, int repeats, cudaStream_t s);
  void run(const cmh_particles &parts, bool want_member, cudaStream_t s);
  // host inputs of nbox boxes: start copying them into input buffer `buf`
  // (after the caller's queued work; every box's positions before any
  // velocities), returning the buffer; take the staged inputs that match
  // `parts` (or copy them now) and return the device descriptions
  int stage_inputs(const cmh_particles *parts, int nbox, cudaStream_t s, int buf);
  std::vector<cmh_particles> take_inputs(const cmh_particles *parts, int nbox, cudaStream_t s);
  // one-buffer mode, after a run's launches are queued: the next staged run's
  // copies, behind the events that say its buffer is free
  void queue_pending();
  void ensure_side();
  void copy_inputs(const cmh_particles *parts, int nbox, int buf, bool behind_run);
};

}  // namespace cmh
