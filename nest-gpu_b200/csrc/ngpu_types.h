// Plain structures shared by the host runtime (ngpu_engine.cpp, ngpu_sim.cpp)
// and the CUDA kernels (ngpu_kernels.cu, ngpu_build.cu): kernel argument
// blocks passed by value.
#pragma once
#include <vector_types.h>

#include <cstdint>

namespace ngpu {

enum Model {
  M_AEIF_COND_BETA = 0,
  M_AEIF_COND_ALPHA,
  M_AEIF_PSC_EXP,
  M_AEIF_PSC_ALPHA,
  M_IAF_PSC_EXP,
  M_SPIKE_GEN,
  M_POISS_GEN,
  M_PARROT,
  M_SPIKE_DET,
  M_NMODEL
};

constexpr int MAX_PORT = 20;          // aeif_*_multisynapse port limit (reference MAX_PORT_NUM)
constexpr int MAX_TPL_PORT = 4;       // port counts with a dedicated kernel instantiation
constexpr int MAX_BATCH = 32;         // time steps per batch at most

// Status bits reported by the device (read back after each Simulate call).
enum Status : unsigned {
  ST_RING_OVERFLOW = 1u << 0,         // more spikes in one step than a ring slot holds
  ST_RK5_TRIALS = 1u << 1,            // RK5 step gave up after the trial cap
  ST_NUMERIC = 1u << 2,               // V_m or w left their guard bounds (reset applied)
  ST_REC_TIMES_FULL = 1u << 3,        // a neuron exceeded its recorded-spike-time capacity
  ST_BARRIER_TIMEOUT = 1u << 4,       // a grid barrier of the persistent step loop gave up waiting
  ST_EXCHANGE_FULL = 1u << 5,         // partitioned network: more local spikes in a batch than the
                                      // exchange buffer holds (the excess was dropped)
};

// Barrier state of the persistent step loop (device memory, zero-initialised).
struct GridBarrier {
  unsigned count;        // blocks arrived at the current barrier
  unsigned gen;          // barriers completed
};

// Simulation clock in device memory.  A CUDA graph covers a fixed number of steps
// split into batches; a kernel of the batch starting at graph step k0 handles the
// per-call steps it = it0 + k0 + m, m < batch length.
struct Clock {
  long long it0;         // per-call index of the first step of the running graph
  long long tidx_base;   // round(t0 / dt): time index of the call's start
  double t0;             // neural time at the call's start [ms]
  long long rec_it0;     // per-call index of the first step of the record window
};

// Spike output context shared by all spiking models.
struct SpikeOut {
  int2 *ring;            // [R][cap] (source node, height bits), slot = time index % R
  int *ring_cnt;         // [R]
  int R, cap;
  const unsigned char *has_out;   // per node: 1 if it has recurrent out-edges to neurons simulated here
  const unsigned char *has_out_all;   // per node: 1 if it has recurrent out-edges anywhere
  // partitioned network: the batch's spikes of the neurons simulated here, for the other
  // processes; xch[0].x counts them, xch[1 + j] = {node, height bits, time index, 0}
  int4 *xch;
  int xch_cap;
  int *last_tidx;        // per node: time index of the most recent spike
  float *last_height;    // per node: height of the most recent spike
  unsigned *status;
  unsigned long long *n_spikes;
  // plastic networks only (else last_rev is null): per node the time index at which its
  // last spike reached its own synapses, set at once (no dendritic delay) or through the
  // reverse ring den_steps[node] steps later
  int *last_rev;
  const int *den_steps;  // [n_nodes] or null (no dendritic delays)
  int *rev_ring;         // [rev_R][rev_cap] nodes whose spike reaches their synapses then
  int *rev_cnt;          // [rev_R]
  int rev_R, rev_cap;
};

// Per-group spike bookkeeping (optional outputs).
struct GroupSpikeRec {
  int *spike_count;      // [n] or null
  int *n_rec;            // [n] or null
  float *rec_times;      // [n * max_rec] or null
  int max_rec;
};

// Record columns of a group, written inside its update kernel before the step's
// input fold (the reference records after the update, src/nestgpu.cu:507).
struct GroupRecord {
  const int *first;      // [n+1] CSR over the group's neurons, or null
  const int2 *col;       // {variable code, column}; code: state index, nvar = refractory
                         // counter, -1 = spike activity
  float *buf;            // [rows][ncol] of the current record window
  int ncol;
};

// Incoming poiss_gen edge, target-major.  Its Poisson stream is keyed by
// (stream, edge_id): edge_id numbers the generator's out-edges in connection order
// (source-major, delay groups ascending, insertion order) from 0, and stream is the
// generator's stream number (its index among all poiss_gen nodes unless set), so a
// generator's draws do not depend on what else the network holds.
struct PoissonIn {
  uint32_t edge_id;
  int gen;               // index into the generator parameter table
  float weight;
  float delay;
  int port;
  uint32_t stream;
};

// Generator parameters: rate [Hz], origin, start, stop [ms].
struct GenPar {
  float rate, origin, start, stop;
};

// Input side of a group: accumulator slots (one per step of a batch) and poiss_gen edges.
struct GroupInput {
  double *acc;           // slot 0 row of this group: acc + m*slot_stride + p*n + i (delivery at
                         // emission: the ring row, slot = time index % PushOut::R)
  size_t slot_stride;    // doubles per slot (all groups)
  const int *pin_off;    // [n+1] or null
  const PoissonIn *pin;
  const GenPar *gen;
  float lam_scale;       // dt / 1000 (rate in Hz -> expected count per step)
  uint64_t seed;
};

// aeif derived parameters: uniform -> value, else a device array.
constexpr int AEIF_NSCAL = 13;
enum AeifPar {
  AP_V_th = 0, AP_Delta_T, AP_inv_Delta_T, AP_g_L, AP_E_L, AP_inv_C_m, AP_a, AP_b,
  AP_inv_tau_w, AP_I_e, AP_V_peak, AP_V_reset, AP_refr_steps
};
// per port: E_rev, inv_t1, inv_t2, port weight
constexpr int AEIF_NPORTPAR = 4;
constexpr int AEIF_NPAR = AEIF_NSCAL + AEIF_NPORTPAR * MAX_PORT;

// Learned step-size context of an aeif group (layouts in ngpu_stepmodel.h).
struct LearnCtx {
  int mode;                       // LearnMode
  float *log;                     // [log_cap][LOG_W] tuples (LM_LOG)
  unsigned long long *log_cursor; // tuples offered so far (may exceed log_cap)
  unsigned long long log_cap;
  const float *model;             // SM_NPAR floats (LM_PROPOSE)
};

struct AeifArgs {
  int n;
  int i0;
  int lo, hi;            // neurons lo .. hi-1 of the group are simulated here (all: 0, n)
  int nport;
  int nvar;
  float *var;            // SoA [nvar][n]: V_m, w, port vars (port-major)
  float *refr;           // [n]
  double *x;             // [n]
  float *h;              // [n]
  GroupInput in;
  GroupRecord rec;
  float dt;
  float hmin;
  float hmin_acc;        // hmin * 1.00001f: forced-accept threshold
  unsigned long long *nderiv;
  int budget;            // RK5 steps per neuron and batch in the main kernel (0: no limit)
  int threads;           // threads per block of the main kernel (64, 128 or 256)
  int occupancy;         // 1: register-capped variant of the main kernel (more resident warps)
  int uniform;           // 1: every parameter is uniform over the group (no parameter arrays)
  int trial_iter;        // 1: main kernel advances one RK5 trial per loop iteration
  int2 *strag_list;      // [n] (neuron, step of the batch) left for the straggler kernel
  int *strag_cnt;        // list length
  GroupSpikeRec srec;
  LearnCtx learn;
  float pval[AEIF_NPAR];
  const float *parr[AEIF_NPAR];
};

enum IafPar {
  IP_I_e = 0, IP_Theta_rel, IP_V_reset_rel, IP_refr_steps, IP_P20, IP_P11ex, IP_P11in,
  IP_P21ex, IP_P21in, IP_P22, IP_NPAR
};

struct IafArgs {
  int n;
  int i0;
  int lo, hi;            // neurons lo .. hi-1 of the group are simulated here (all: 0, n)
  float *var;            // SoA [4][n]: I_syn_ex, I_syn_in, V_m_rel, refractory_step
  GroupInput in;
  GroupRecord rec;
  float dt;
  GroupSpikeRec srec;
  float pval[IP_NPAR];
  const float *parr[IP_NPAR];
};

// parrot_neuron (src/parrot_neuron.cu:40-130): vars input_spike_height, dummy_input, V.
struct ParrotArgs {
  int n;
  int i0;
  int lo, hi;            // neurons lo .. hi-1 of the group are simulated here (all: 0, n)
  float *var;            // SoA [3][n]
  const float *hold;     // [n] hold_spike_height
  GroupInput in;
  GroupRecord rec;
  float dt;
  GroupSpikeRec srec;
};

struct SpikeGenArgs {
  int n;
  int i0;
  int lo, hi;            // neurons lo .. hi-1 of the group are simulated here (all: 0, n)
  const int *off;        // [n+1] into tidx/height
  const int *tidx;       // spike step indices (per-call step counter)
  const float *height;
  int *next;             // [n]
  GroupRecord rec;
  float dt;
  GroupSpikeRec srec;
};

// Recurrent edge: packed accumulator index (receptor row + target) and weight.
struct EdgeW {
  uint32_t acc;
  float w;
};

// Delivery at emission (networks of iaf_psc_exp groups): the update kernel's block adds each
// spike's out-edges at once into the accumulator ring acc[R][stride], slot = arrival time
// index % R; the spike ring is then not used.
struct PushOut {
  double *acc;
  int R;
  size_t stride;
  const long long *ev_off;   // delivery CSR [n_nodes * dspan + 1]
  const EdgeW *edge;
  int dmin, dspan;
  unsigned long long *n_events;
};

struct DeliverArgs {
  const int2 *ring;
  int *ring_cnt;
  int R, cap;
  int dmin, dspan;       // delay indices dmin .. dmin+dspan-1
  const long long *ev_off;   // [n_nodes * dspan + 1]
  const EdgeW *edge;
  double *acc;           // slot 0
  size_t slot_stride;
  float dt;
  unsigned long long *n_events;
  int *strag_cnt;        // per-group straggler counters, cleared for the batch
  int n_strag;
  int aggregate;         // 1 (with 32-lane groups): warp-aggregated reductions
  int prefetch;          // 1: the next work item's ring entry and offsets loaded ahead
  int4 *xch;             // partitioned network: exchange buffer whose count the batch clears
};

// Plastic edge (synapse group > 0): its position in the delivery CSR, its target node and
// its synapse group (1-based).  Forward order: by (source, delay) segment, insertion order
// inside a segment.
struct PlasticEdge {
  unsigned long long pos;
  int target;
  int group;
};

constexpr int SYN_NPAR = 8;   // parameter slots per synapse group (stdp uses 7)
enum SynType { SYN_TEST = 0, SYN_STDP = 1 };

// Spike-timing-dependent plasticity, one time step per batch (src/get_spike.cu:85-95,
// src/rev_spike.cu:46-130).
struct StdpArgs {
  const int2 *ring;
  const int *ring_cnt;
  int R, cap;
  int dmin, dspan;
  const int *pl_off;          // [n_nodes * dspan + 1] plastic entries per (source, delay) segment
  const PlasticEdge *pl;      // [n_pl]
  unsigned short *stamp;      // [n_pl] low 16 bits of the time index of the last arrival
  long long n_pl;
  EdgeW *edge;                // delivery CSR (weights updated in place)
  const int *last_tidx;       // per node: time index of its last spike, -1 before the first
  const int *syn_type;        // [n_groups]
  const float *syn_par;       // [n_groups][SYN_NPAR]
  const int *rev_off;         // [n_rev_nodes + 1] into rev_id
  const int *rev_id;          // plastic entries grouped by target
  const int *rev_node;        // [n_rev_nodes] targets with plastic in-edges
  int n_rev_nodes;
  float dt;
};

// Generated connection block: fixed in-degree with per-target random sources
// and uniform delays, drawn on the device (see ngpu_build.cu).
struct GenBlockDev {
  int src0, nsrc, ntgt, k;
  int tgt_i0_rel;          // first target relative to its group
  int group_n;             // targets' group size
  unsigned long long acc_base;   // accumulator offset of the targets' group + port row
  float w;
  int dlo, dhi;            // delay indices, inclusive
  uint64_t seed;
  int t_begin, t_end;      // block-relative targets whose edges are generated here
};

// A rule-based connection call (src/connect_rules.h:161-338) whose edges are expanded on the
// device at calibration.  The random numbers are the call's cuRAND draws, kept on the device:
//   rule 2 (fixed_total_number): edge i: source index rnd[2i] % ns, target index rnd[2i+1] % nt,
//          array index i;
//   rule 3 (fixed_indegree): edge (kk, i): source index pick[i], target index kk, array index
//          kk * degree + i;
//   rule 4 (fixed_outdegree): edge (kk, i): source index kk, target index pick[i], array index
//          kk * degree + i.
// An index j maps to node src_arr[j] (or src0 + j), likewise for targets.
struct RuleBlockDev {
  int rule;
  int ns, nt, degree, port;
  int src0, tgt0;
  const int *src_arr, *tgt_arr;   // node arrays or null (contiguous ranges)
  const unsigned *rnd;            // rule 2: 2 * degree draws
  const int *pick;                // rules 3, 4: degree picks shared by all targets (sources)
  float w, d_ms;                  // uniform weight and delay [ms] ...
  const float *warr, *darr;       // ... or per-edge arrays
  long long n_edges;
  float dt;
};

}  // namespace ngpu
