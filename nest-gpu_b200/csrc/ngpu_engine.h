// Host runtime of the spiking engine: node groups with structure-of-arrays
// state, the connection store and rules, calibration into the device layout
// (CSR by (source, delay), target-major poiss_gen edges, spike ring), and the
// CUDA-graph step loop.  One process-wide instance sits behind the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <curand.h>

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "ngpu_stepmodel.h"
#include "ngpu_types.h"

namespace ngpu {

// Error with the reference's C-ABI code 2 (ngpu_exception).
struct NgpuError : public std::runtime_error {
  explicit NgpuError(const std::string &m) : std::runtime_error(m) {}
};

// Training of the learned step-size proposal.
struct TrainConfig {
  long long iters = 3000;        // Adam iterations
  int batch = 4096;              // samples per iteration (multiple of 128)
  float lr = 2.0e-3f;
  float safety = 0.9f;           // proposal = safety * predicted step size
  float floor = 0.0f;            // proposal >= floor * controller h (0: no floor)
  uint64_t seed = 1;
};
struct TrainResult {
  long long n_used = 0;          // logged tuples the network is trained on
  float final_loss = 0.0f;       // mean squared error (normalised target), last iterations
};
TrainResult train_step_model(const float *d_tuples, long long n_tuples, const TrainConfig &cfg, float *params);
void mlp_forward_host(const float *params, const float *feat, int n, float *out);
void mlp_grad_host(const float *params, const float *feat, const float *target, int n, float *grad, float *loss);
void set_tensor_wait_test(int on);

// Kinds of named quantities of a node group.
enum Kind { K_NONE = -1, K_SCAL_VAR = 0, K_PORT_VAR, K_SCAL_PARAM, K_PORT_PARAM, K_GROUP_PARAM,
            K_ARRAY_PARAM, K_INT_VAR };

struct Group {
  int model = 0;
  int i0 = 0, n = 0, nport = 0;
  // user-visible parameters [param][neuron] (scalar params then port params port-major)
  std::vector<std::vector<float>> par;
  // state variables [var][neuron]: authoritative on the host until calibration
  std::vector<std::vector<float>> var;
  float h_min_rel = 1.0e-3f, h0_rel = 1.0e-2f;
  // spike_generator
  std::vector<std::vector<float>> sg_times, sg_heights;
  // recording options
  bool spike_count_on = false;
  int max_rec = 0;
  int rec_times_step = 0;
  std::vector<std::vector<float>> rec_times_host;   // drained, not yet handed out
  std::vector<std::vector<float>> rec_export;       // handed out by the last query
  std::vector<int> rec_n_host;                   // exported counts
  std::vector<float *> rec_ptr_host;             // exported row pointers
  // device state
  float *d_var = nullptr;        // [nvar][n]
  float *d_hold = nullptr;       // parrot_neuron: hold_spike_height [n]
  float *d_refr = nullptr;       // aeif refractory counter
  double *d_x = nullptr;
  float *d_h = nullptr;
  size_t acc_off = 0;
  std::vector<float *> d_der;    // derived-parameter arrays (null = uniform)
  std::vector<float> der_val;    // derived-parameter uniform values
  int *d_spike_count = nullptr;
  int *d_n_rec = nullptr;
  float *d_rec_times = nullptr;
  int2 *d_strag = nullptr;       // aeif: straggler list [n] (neuron, step of the batch)
  int strag_slot = -1;           // index of its counter in the engine's counter array
  int *d_rec_first = nullptr;    // record columns: CSR over neurons
  int2 *d_rec_col = nullptr;
  int *d_pin_off = nullptr;
  PoissonIn *d_pin = nullptr;
  int *d_sg_off = nullptr, *d_sg_tidx = nullptr, *d_sg_next = nullptr;
  float *d_sg_h = nullptr;
  int lo = 0, hi = 0;            // neurons lo .. hi-1 are simulated by this process (calibration)
  int gen0 = -1;                 // poiss_gen: first row in the generator table
  std::vector<uint32_t> pg_stream;   // poiss_gen: stream numbers (empty: index among generators)
  bool dirty = true;             // parameters changed since last upload
};

struct RecordSpec {
  std::string file;
  std::vector<std::string> var;
  std::vector<int> node, port;
  std::vector<std::vector<float>> data;
  std::vector<float *> row_ptr;
  FILE *fp = nullptr;
};

struct EngineStats {
  unsigned long long n_derivs = 0;      // RK5 derivative evaluations
  unsigned long long n_events = 0;      // synaptic events delivered
  unsigned long long n_spikes = 0;
  double sim_seconds = 0.0;             // wall time inside the step loop of the last Simulate
  double sim_device_ms = 0.0;           // device time (CUDA events) of the last Simulate
  long long steps = 0;
  unsigned status = 0;
};

class Engine {
 public:
  Engine();
  ~Engine();

  // ---- kernel settings (src/nestgpu.cu:64-99, 1705-1947)
  float dt = 0.1f;
  unsigned long long seed = 54321ULL;
  unsigned long long kernel_seed = 54321ULL + 12345ULL;
  int max_spike_buffer_size = 20;
  int verbosity = 4;
  bool print_time = false;
  float max_spike_num_fact = 1.0f;
  float max_spike_per_host_fact = 1.0f;
  int remote_spike_height = 0;
  float sim_time = 1000.0f;
  int graph_steps = 100;          // steps per captured CUDA graph
  int rk5_budget = 4;             // RK5 steps per neuron before the straggler kernel takes over
  int deliver_blocks_req = 0;     // delivery grid size (0: from the number of spiking sources)
  int batch_max = MAX_BATCH;      // upper bound of the time-batch length (1: step by step)
  int update_threads = 128;       // threads per block of the aeif update kernel (64, 128, 256)
  int deliver_group = 32;         // lanes per delivery work item (8, 16, 32)
  int deliver_aggregate = 0;      // 1: warp-aggregated reductions (with 32-lane work items)
  int deliver_prefetch = 0;       // 1: delivery loads the next work item's segment ahead
  int deliver_push = 0;           // 1: networks of iaf_psc_exp groups deliver each spike at emission
                                  // (set before calibration)
  int update_occupancy = 0;       // 1: register-capped aeif update kernel
  int update_trial_iter = 0;      // 1: aeif update kernel advances one RK5 trial per iteration
  int persistent = 0;             // iaf-only networks: persistent cooperative step loop
  int launch_pdl = -1;            // programmatic dependent launch of the batch kernels (-1: one-step batches)
  int barrier_extra = 0;          // test hook: blocks the persistent loop's barriers wait for in excess
  bool use_device_rng = true;     // cuRAND device generator (as the reference) if a GPU exists

  // ---- one network over several processes (one GPU each): process `rank` of `world`
  //      simulates a contiguous share of every node group; after each time batch the spikes
  //      of its neurons are handed to `exchange` (see set_exchange)
  void set_partition(int rank, int world);
  // send / recv: device buffers of int4 records, (cap + 1) per process (recv holds world
  // blocks, block q = process q's send buffer); exchange(user) must fill recv from every
  // process's send buffer (an all-gather) and return 0 once recv may be read
  void set_exchange(void *send, void *recv, long long cap, int (*exchange)(void *), void *user);
  int part_rank() const { return part_rank_; }
  int part_world() const { return part_world_; }

  void set_seed(unsigned long long s);
  void set_time_resolution(float t);

  // ---- nodes
  int create(const std::string &model, int n, int nport);
  int create_poisson_generator(int n, float rate);
  Group &group_of(int node);
  int group_index(int node);
  int n_nodes() const { return (int)node_group_.size(); }
  Kind locate(int node, const std::string &name, int *idx = nullptr);
  std::vector<std::string> names(int node, Kind k);
  int param_size(int node, const std::string &name);
  int var_size(int node, const std::string &name);

  void set_scalar(const std::vector<int> &nodes, const std::string &name, float v);
  void set_port_or_array(const std::vector<int> &nodes, const std::string &name, const float *a, int sz);
  void set_int_var(const std::vector<int> &nodes, const std::string &name, int v);
  std::vector<float> get_values(const std::vector<int> &nodes, const std::string &name);   // node-major
  std::vector<int> get_int_values(const std::vector<int> &nodes, const std::string &name);
  // nodes i0 .. i0+n-1 of one group, copied straight into out (n ints)
  void get_int_values_seq(int i0, int n, const std::string &name, int *out);
  std::vector<float> get_array_param(int node, const std::string &name);
  void set_group_param(const std::vector<int> &nodes, const std::string &name, float v);
  float get_group_param(int node, const std::string &name);

  // ---- random numbers (cuRAND, as src/random.cu:8-76)
  std::vector<unsigned> random_int(size_t n);
  std::vector<float> random_uniform(size_t n);
  std::vector<float> random_normal(size_t n, float mean, float sd);
  std::vector<float> random_normal_clipped(size_t n, float mean, float sd, float vmin, float vmax,
                                           float vstep);

  // ---- synapse groups (src/syn_model.cu:136-238): 1-based, 0 is the static synapse
  int create_syn_group(const std::string &model);
  std::vector<std::string> syn_group_param_names(int g) const;
  int syn_group_param_idx(int g, const std::string &name) const;
  float get_syn_group_param(int g, const std::string &name) const;
  void set_syn_group_param(int g, const std::string &name, float v);

  // ---- connections
  void connect1(int src, int tgt, int port, int syn_group, float w, float d);
  void connect_rule(int rule, const int *src_arr, int src0, int ns, const int *tgt_arr, int tgt0,
                    int nt, int degree, int port, int syn_group, float w, float d,
                    const float *warr, const float *darr);
  size_t n_connections() const { return c_src_.size() + n_generated_ + n_rule_edges_; }
  // rule-based calls with at least this many edges are expanded on the device (a device
  // cuRAND generator is needed); smaller ones go to the host store at once
  long long device_rule_min_edges = 1LL << 16;
  // ids (source, group, index) in reference order, filtered (syn_group < 0: any group)
  std::vector<int> get_connections(const int *src_arr, int src0, int ns, const int *tgt_arr,
                                   int tgt0, int nt, int syn_group = -1);
  void connection_status(int src, int grp, int idx, int *tgt, unsigned char *port,
                         unsigned char *syn, float *delay, float *w);
  // Bulk import of a prebuilt edge list (engine extension, used by the large benchmarks).
  void connect_arrays(size_t n, const int *src, const int *tgt, const unsigned char *port,
                      const float *w, const float *d);
  // poiss_gen nodes i0 .. i0+n-1 draw from streams stream0 .. stream0+n-1 (engine extension)
  void set_poisson_stream(int i0, int n, uint32_t stream0);
  void connect_fixed_indegree_per_target(int src0, int ns, int tgt0, int nt, int k, int port,
                                         float w, float dmin_ms, float dmax_ms, uint64_t seed);

  // ---- recording
  int create_record(const std::string &file, const std::vector<std::string> &vars,
                    const std::vector<int> &nodes, const std::vector<int> &ports);
  RecordSpec &record(int i);
  void activate_spike_count(int i_node, int n);
  void activate_rec_spike_times(int i_node, int n, int max_n);
  void set_rec_spike_times_step(int i_node, int n, int step);
  int n_rec_spike_times(int node);
  void get_rec_spike_times(int i_node, int n, int **n_pt, float ***t_pt);

  // ---- simulation
  void calibrate();
  void simulate(float t);
  void start_simulation();
  void simulation_step();
  void end_simulation();
  bool calibrated() const { return calibrated_; }
  bool push_active() const { return push_; }   // delivery at emission (set at calibration)
  double neural_time() const { return neural_time_; }
  EngineStats stats();
  // Run n steps with every kernel bracketed by CUDA events on the engine stream;
  // returns the average device time per step [ms] of: neuron updates (all groups),
  // record gather, spike delivery.  The steps are ordinary simulation steps.
  std::vector<double> profile_steps(int n);
  // The recurrent delivery layout after calibration: segments by (source node, delay step
  // - dmin), nodes * dspan + 1 offsets, and per edge its target node, receptor port, weight.
  void delivery_shape(int *n_nodes, int *dmin, int *dspan, long long *n_edges);
  void delivery_csr(long long *seg_off, int *target, unsigned char *port, float *weight);
  long long n_launches() const { return n_launch_; }

  // Tune update_threads, update_occupancy, deliver_group, deliver_blocks_req and rk5_budget
  // (and the persistent loop where eligible) on the calibrated network: after 4 x `steps`
  // warm-up steps, each candidate is timed twice over `steps` simulation steps (coordinate
  // descent, two passes).  The trials are ordinary simulation steps: the network advances
  // by them.  Returns the number of trials; the chosen values stay set.
  int autotune(int steps, std::vector<std::pair<std::string, double>> *log);

  // ---- learned RK5 step-size proposal (kernels and training in ngpu_learn.cu)
  // Log one tuple per accepted RK5 step of every aeif neuron (at most cap tuples).
  void rk5_log_start(long long cap);
  void rk5_log_stop();
  long long rk5_log_count(long long *offered);
  void rk5_log_get(float *out, long long first, long long n);
  // Train the proposal network on the logged tuples with the GPU kernels; the
  // result becomes the engine's model.
  TrainResult step_model_train(const TrainConfig &cfg);
  void step_model_set(const float *p);
  void step_model_get(float *p) const;
  bool has_step_model() const { return has_model_; }
  void step_model_enable(bool on);
  // Analysis mode: every RK5 step starts from the largest step that passes the unchanged
  // error test (the search is not counted), the floor of evaluations for any proposal.
  void step_bound_mode(bool on);
  int learn_mode() const { return learn_mode_; }
  int batch_length() const { return batch_; }
  // captured graphs hold the launch mappings: drop them when a mapping knob changes
  void invalidate_graphs();

  // device buffers exposed to the engine-level helpers
  cudaStream_t stream() const { return stream_; }

 private:
  std::vector<Group> groups_;
  std::vector<int> node_group_;
  std::vector<RecordSpec> records_;
  // connection store, insertion order
  std::vector<int> c_src_, c_tgt_;
  std::vector<unsigned char> c_port_;
  std::vector<float> c_w_;
  std::vector<int> c_d_;
  std::vector<unsigned char> c_syn_;   // synapse group per edge; empty while all are static
  unsigned char syn_of(size_t e) const { return c_syn_.empty() ? 0 : c_syn_[e]; }
  struct SynGroupDef {
    int type;                 // SynType
    std::vector<float> par;
  };
  std::vector<SynGroupDef> syn_groups_;
  // generated blocks (connect_fixed_indegree_per_target)
  struct GenBlock {
    int src0, nsrc, tgt0, ntgt, k, port;
    float w, dmin_ms, dmax_ms;
    uint64_t seed;
  };
  std::vector<GenBlock> blocks_;
  size_t n_generated_ = 0;
  // rule-based calls expanded on the device at calibration (RuleBlockDev): their random
  // numbers and arrays stay on the device; the host store gets their edges only when a
  // query needs them (materialize_rule_blocks), spliced in at their place in call order
  struct RuleBlock {
    size_t host_pos;                 // host-store edges inserted before the call
    RuleBlockDev dev;                // device pointers (engine allocations)
    std::vector<int> src_arr, tgt_arr;   // host copies of node arrays (empty: ranges)
    int dlo, dhi;                    // delay-step range of the call's edges
  };
  std::vector<RuleBlock> rblocks_;
  size_t n_rule_edges_ = 0;
  bool connect_rule_device(int rule, const int *src_arr, int src0, int ns, const int *tgt_arr, int tgt0,
                           int nt, int degree, int port, float w, float d, const float *warr,
                           const float *darr);
  void materialize_rule_blocks();
  template <class T> T *dcopy(const T *h, size_t n);
  // reference order cache: permutation, group index and index-in-group per edge
  bool order_valid_ = false;
  std::vector<long long> ord_;          // edge ids in reference order
  std::vector<long long> src_first_;    // per source: first position in ord_
  std::vector<int> ord_grp_, ord_idx_;  // per position
  void build_order();

  curandGenerator_t gen_ = nullptr;
  bool gen_device_ = false;
  void make_generator();

  // simulation state
  bool calibrated_ = false;
  bool first_sim_ = true;
  bool in_sim_ = false;
  double neural_time_ = 0.0;
  double neur_t0_ = 0.0;
  long long it_ = 0, Nt_ = 0;
  long long tidx_base_ = 0;

  // device
  cudaStream_t stream_ = nullptr;
  cudaStream_t stream2_ = nullptr;      // second stream for non-aeif groups (fork / join per batch)
  // plastic edges (synapse groups): forward index by (source, delay), reverse by target
  bool plastic_ = false;
  StdpArgs stdp_{};
  int *d_last_rev_ = nullptr;      // plastic networks: last spike arrival at each node's synapses
  int *d_den_steps_ = nullptr;     // dendritic delays in steps (null when all are 0)
  int *d_rev_ring_ = nullptr, *d_rev_cnt_ = nullptr;
  int rev_R_ = 0, rev_cap_ = 0;
  std::vector<unsigned long long> pl_pos_;               // per plastic entry: CSR position
  std::vector<std::pair<size_t, int>> pl_of_edge_;       // (host edge, plastic entry), sorted
  void build_plastic(const std::vector<size_t> &pl_edge, const std::vector<long long> &pl_key,
                     const std::vector<int> &pl_rank);
  void upload_syn_groups();
  float plastic_weight(size_t e, float fallback);
  cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
  Clock *d_clk_ = nullptr;
  double *d_acc_ = nullptr;
  size_t n_acc_ = 0;
  bool push_ = false;             // delivery at emission is active (chosen at calibration)
  double *d_pacc_ = nullptr;      // its accumulator ring [push_R_][n_acc_]
  int push_R_ = 0;
  int2 *d_ring_ = nullptr;
  int *d_ring_cnt_ = nullptr;
  int R_ = 0, cap_ = 0;
  unsigned char *d_has_out_ = nullptr;
  int *d_last_tidx_ = nullptr;
  float *d_last_h_ = nullptr;
  unsigned *d_status_ = nullptr;
  long long *d_ev_off_ = nullptr;
  EdgeW *d_edge_ = nullptr;
  size_t n_edge_dev_ = 0;
  int dmin_ = 0, dspan_ = 1;
  GenPar *d_gen_ = nullptr;
  int n_gen_ = 0;
  unsigned long long *d_counters_ = nullptr;   // [0] derivs, [1] events
  float *d_recbuf_ = nullptr;
  int rec_ncol_ = 0, rec_rows_cap_ = 0;
  int batch_ = 1;                // steps per batch
  int *d_strag_cnt_ = nullptr;   // straggler counters, one per aeif group
  int n_strag_ = 0;
  int deliver_blocks_ = 148;
  std::map<int, cudaGraphExec_t> graphs_;
  std::vector<void *> allocs_;
  double last_sim_seconds_ = 0.0;
  double last_sim_device_ms_ = 0.0;
  long long n_launch_ = 0;                 // kernels launched (graph replays count their nodes)
  std::map<int, long long> graph_nodes_;   // kernels per captured graph
  bool capturing_ = false;
  long long capture_count_ = 0;
  void count_launch(long long n) { if (capturing_) capture_count_ += n; else n_launch_ += n; }
  cudaEvent_t ev_a_ = nullptr, ev_b_ = nullptr;
  long long total_steps_ = 0;
  unsigned status_seen_ = 0;
  // learned step size
  int learn_mode_ = 0;
  float *d_log_ = nullptr;
  unsigned long long *d_log_cursor_ = nullptr;
  long long log_cap_ = 0;
  float *d_model_ = nullptr;
  std::vector<float> model_;
  bool has_model_ = false;
  void set_learn_mode(int mode);
  // all iaf_psc_exp groups in one launch when there are several
  IafArgs *d_iaf_tab_ = nullptr;
  int *d_iaf_blk0_ = nullptr;
  int *d_iaf_first_ = nullptr;   // neuron prefix over the iaf groups
  GridBarrier *d_bar_ = nullptr;
  int n_iaf_multi_ = 0, iaf_multi_blocks_ = 0;
  void prepare_multi();
  bool persistent_eligible() const;
  bool push_eligible() const;
  void run_persistent(int steps);

  template <class T> T *dalloc(size_t n);
  void free_device();
  void upload_params();
  void upload_dirty_params();   // upload_params() if any group's parameters changed
  void build_records();
  void launch_batch(int k0, int M, std::vector<cudaEvent_t> *ev);
  void ensure_record_window(long long rows);
  GroupRecord group_record(Group &g);
  GroupInput group_input(Group &g);
  void run_steps(long long n);
  void run_batches_partitioned(long long n);
  int part_rank_ = 0, part_world_ = 1;
  int4 *xch_send_ = nullptr, *xch_recv_ = nullptr;
  int xch_cap_ = 0;
  int (*xch_fn_)(void *) = nullptr;
  void *xch_user_ = nullptr;
  unsigned char *d_has_out_all_ = nullptr;
  void drain_records(long long rows);
  void drain_rec_spike_times();
  SpikeOut spike_out() const;
  PushOut push_out() const;
  AeifArgs aeif_args(Group &g);
  IafArgs iaf_args(Group &g);
  SpikeGenArgs sg_args(Group &g);
  ParrotArgs parrot_args(Group &g);
  DeliverArgs deliver_args();
  void check_status();
};

Engine &engine();
void engine_reset();

// launchers (ngpu_kernels.cu)
int launch_aeif(int model, const AeifArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M,
                cudaStream_t st);
int launch_iaf(const IafArgs &A, const SpikeOut &so, const PushOut *po, const Clock *clk, int k0, int M,
               cudaStream_t st);
int launch_iaf_multi(const IafArgs *tab, const int *blk0, int ngroups, int nblocks, const SpikeOut &so,
                     const PushOut *po,
                     const Clock *clk, int k0, int M, cudaStream_t st);
int launch_spike_gen(const SpikeGenArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M,
                     cudaStream_t st);
int launch_parrot(const ParrotArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M, cudaStream_t st);
int launch_spike_det(const ParrotArgs &A, const SpikeOut &so, const Clock *clk, int k0, int M, cudaStream_t st);
int launch_rev_arrivals(int *rev_ring, int *rev_cnt, int rev_R, int rev_cap, int *last_rev, const Clock *clk,
                        int k0, cudaStream_t st);
int launch_deliver(const DeliverArgs &A, int n_blocks, int group, const Clock *clk, int k0, int M,
                   cudaStream_t st);
int launch_clock_advance(Clock *clk, int K, cudaStream_t st);
int launch_exchange_unpack(const SpikeOut &so, const int4 *recv, int xch_cap, int world, int rank,
                           cudaStream_t st);
void mark_sources_device(const std::vector<GenBlockDev> &blocks, const std::vector<RuleBlockDev> &rblocks,
                         unsigned char *d_flag, cudaStream_t st);
void set_launch_pdl(bool on);
// reduction-rate probe (ngpu_probe.cu): 1e9 random FP64 reductions per second
double measure_random_reduction_rate(size_t bytes, long long n_ops);
// STDP (ngpu_stdp.cu)
int launch_stdp_reset(const StdpArgs &A, const Clock *clk, int k0, cudaStream_t st);
int launch_stdp_forward(const StdpArgs &A, const Clock *clk, int k0, cudaStream_t st);
int launch_stdp_reverse(const StdpArgs &A, const Clock *clk, int k0, cudaStream_t st);
int launch_persistent_iaf(const DeliverArgs &D, int group, const IafArgs *tab, const int *first, int ngroups,
                          const SpikeOut &so, const Clock *clk, int steps, int M, GridBarrier *bar, int max_blocks,
                          int barrier_extra, cudaStream_t st);
int deliver_max_pairs();
void pack_delivery_csr_noalloc(const int *src, const int *dly, const unsigned *target, const float *weight,
                               size_t n, int n_nodes, int dspan, unsigned long long *seg_off, EdgeW *edge,
                               cudaStream_t st);
void pack_delivery_csr(const int *src, const int *dly, const unsigned *target, const float *weight,
                       size_t n, int n_nodes, int dspan, unsigned long long *seg_off, EdgeW *edge,
                       cudaStream_t st);
void build_csr_device(int n_nodes, int dmin, int dspan, const std::vector<int> &cnt_host,
                      const std::vector<long long> &h_key, const std::vector<int> &h_rank,
                      const std::vector<EdgeW> &h_ew, const std::vector<GenBlockDev> &blocks,
                      const std::vector<RuleBlockDev> &rblocks, const unsigned *d_node_acc0,
                      const int *d_node_gn, unsigned long long **d_off_out, EdgeW **d_edge_out,
                      size_t *n_edge_out, unsigned char *d_has_out, cudaStream_t st);

}  // namespace ngpu
