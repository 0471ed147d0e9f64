/*
 * nestgpu_b200.h -- C ABI of the B200 spiking engine (libnestgpu_b200.so).
 *
 * The NESTGPU_* entry points have exactly the names, argument types and
 * meaning of the reference's C ABI (NEST GPU 1.08, src/nestgpu_C.h); the line
 * cited beside each group is where the reference declares the function this
 * one replaces.  A program bound to the reference library (pythonlib/nestgpu.py
 * loads it with ctypes through NESTGPU_LIB) binds to this one unchanged.
 *
 * Conventions shared with the reference:
 *  - every call first clears the error state; on failure it sets an error code
 *    (2: engine error, 1: allocation failure, 255: other) and a message, read
 *    with NESTGPU_GetErrorCode / NESTGPU_GetErrorMessage;
 *  - NESTGPU_SetOnException(0) (the default) makes a failing call print the
 *    message and exit the process with the code; 1 returns to the caller;
 *  - getters return host arrays the caller owns (malloc'd), except
 *    NESTGPU_GetRecordData and NESTGPU_GetRecSpikeTimes, which point into
 *    engine-owned storage valid until the next call of the same function.
 *  - MPI entry points exist for binary compatibility: one process, rank 0.
 *
 * Entry points prefixed NGPU_ are engine extensions with no counterpart in
 * the reference; each says so.
 */
#ifndef NESTGPU_B200_H
#define NESTGPU_B200_H

#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* errors, seeds, kernel settings: src/nestgpu_C.h:34-52 */
char *NESTGPU_GetErrorMessage();
unsigned char NESTGPU_GetErrorCode();
void NESTGPU_SetOnException(int on_exception);
int NESTGPU_SetRandomSeed(unsigned long long seed);
int NESTGPU_SetTimeResolution(float time_res);
float NESTGPU_GetTimeResolution();
int NESTGPU_SetMaxSpikeBufferSize(int max_size);
int NESTGPU_GetMaxSpikeBufferSize();
int NESTGPU_SetSimTime(float sim_time);
int NESTGPU_SetVerbosityLevel(int verbosity_level);

/* node creation and records: src/nestgpu_C.h:54-66 */
int NESTGPU_Create(char *model_name, int n_neuron, int n_port);
int NESTGPU_CreatePoissonGenerator(int n_node, float rate);
int NESTGPU_CreateRecord(char *file_name, char *var_name_arr[], int *i_node_arr, int *port_arr,
                         int n_node);
int NESTGPU_GetRecordDataRows(int i_record);
int NESTGPU_GetRecordDataColumns(int i_record);
float **NESTGPU_GetRecordData(int i_record);

/* parameters and variables: src/nestgpu_C.h:68-141 */
int NESTGPU_SetNeuronScalParam(int i_node, int n_neuron, char *param_name, float val);
int NESTGPU_SetNeuronArrayParam(int i_node, int n_neuron, char *param_name, float *param,
                                int array_size);
int NESTGPU_SetNeuronPtScalParam(int *i_node, int n_neuron, char *param_name, float val);
int NESTGPU_SetNeuronPtArrayParam(int *i_node, int n_neuron, char *param_name, float *param,
                                  int array_size);
int NESTGPU_IsNeuronScalParam(int i_node, char *param_name);
int NESTGPU_IsNeuronPortParam(int i_node, char *param_name);
int NESTGPU_IsNeuronArrayParam(int i_node, char *param_name);
int NESTGPU_SetNeuronIntVar(int i_node, int n_neuron, char *var_name, int val);
int NESTGPU_SetNeuronScalVar(int i_node, int n_neuron, char *var_name, float val);
int NESTGPU_SetNeuronArrayVar(int i_node, int n_neuron, char *var_name, float *var, int array_size);
int NESTGPU_SetNeuronPtIntVar(int *i_node, int n_neuron, char *var_name, int val);
int NESTGPU_SetNeuronPtScalVar(int *i_node, int n_neuron, char *var_name, float val);
int NESTGPU_SetNeuronPtArrayVar(int *i_node, int n_neuron, char *var_name, float *var,
                                int array_size);
int NESTGPU_IsNeuronIntVar(int i_node, char *var_name);
int NESTGPU_IsNeuronScalVar(int i_node, char *var_name);
int NESTGPU_IsNeuronPortVar(int i_node, char *var_name);
int NESTGPU_IsNeuronArrayVar(int i_node, char *var_name);
int NESTGPU_GetNeuronParamSize(int i_node, char *param_name);
int NESTGPU_GetNeuronVarSize(int i_node, char *var_name);
float *NESTGPU_GetNeuronParam(int i_node, int n_neuron, char *param_name);
float *NESTGPU_GetNeuronPtParam(int *i_node, int n_neuron, char *param_name);
float *NESTGPU_GetArrayParam(int i_node, char *param_name);
int *NESTGPU_GetNeuronIntVar(int i_node, int n_neuron, char *param_name);
int *NESTGPU_GetNeuronPtIntVar(int *i_node, int n_neuron, char *param_name);
float *NESTGPU_GetNeuronVar(int i_node, int n_neuron, char *param_name);
float *NESTGPU_GetNeuronPtVar(int *i_node, int n_neuron, char *param_name);
float *NESTGPU_GetArrayVar(int i_node, char *var_name);

/* simulation control: src/nestgpu_C.h:143-151 */
int NESTGPU_Calibrate();
int NESTGPU_Simulate();
int NESTGPU_StartSimulation();
int NESTGPU_SimulationStep();
int NESTGPU_EndSimulation();

/* MPI (single process: rank 0 of 1): src/nestgpu_C.h:153-161 */
int NESTGPU_ConnectMpiInit(int argc, char *argv[]);
int NESTGPU_MpiId();
int NESTGPU_MpiNp();
int NESTGPU_ProcMaster();
int NESTGPU_MpiFinalize();

/* random numbers from the connection generator: src/nestgpu_C.h:163-170 */
unsigned int *NESTGPU_RandomInt(size_t n);
float *NESTGPU_RandomUniform(size_t n);
float *NESTGPU_RandomNormal(size_t n, float mean, float stddev);
float *NESTGPU_RandomNormalClipped(size_t n, float mean, float stddev, float vmin, float vmax,
                                   float vstep);

/* connections: src/nestgpu_C.h:172-222 */
int NESTGPU_Connect(int i_source_node, int i_target_node, unsigned char port,
                    unsigned char syn_group, float weight, float delay);
int NESTGPU_ConnSpecInit();
int NESTGPU_SetConnSpecParam(char *param_name, int value);
int NESTGPU_ConnSpecIsParam(char *param_name);
int NESTGPU_SynSpecInit();
int NESTGPU_SetSynSpecIntParam(char *param_name, int value);
int NESTGPU_SetSynSpecFloatParam(char *param_name, float value);
int NESTGPU_SetSynSpecFloatPtParam(char *param_name, float *array_pt);
int NESTGPU_SynSpecIsIntParam(char *param_name);
int NESTGPU_SynSpecIsFloatParam(char *param_name);
int NESTGPU_SynSpecIsFloatPtParam(char *param_name);
int NESTGPU_ConnectSeqSeq(int i_source, int n_source, int i_target, int n_target);
int NESTGPU_ConnectSeqGroup(int i_source, int n_source, int *i_target, int n_target);
int NESTGPU_ConnectGroupSeq(int *i_source, int n_source, int i_target, int n_target);
int NESTGPU_ConnectGroupGroup(int *i_source, int n_source, int *i_target, int n_target);
int NESTGPU_RemoteConnectSeqSeq(int i_source_host, int i_source, int n_source, int i_target_host,
                                int i_target, int n_target);
int NESTGPU_RemoteConnectSeqGroup(int i_source_host, int i_source, int n_source,
                                  int i_target_host, int *i_target, int n_target);
int NESTGPU_RemoteConnectGroupSeq(int i_source_host, int *i_source, int n_source,
                                  int i_target_host, int i_target, int n_target);
int NESTGPU_RemoteConnectGroupGroup(int i_source_host, int *i_source, int n_source,
                                    int i_target_host, int *i_target, int n_target);

/* names: src/nestgpu_C.h:224-254 */
char **NESTGPU_GetIntVarNames(int i_node);
char **NESTGPU_GetScalVarNames(int i_node);
int NESTGPU_GetNIntVar(int i_node);
int NESTGPU_GetNScalVar(int i_node);
char **NESTGPU_GetPortVarNames(int i_node);
int NESTGPU_GetNPortVar(int i_node);
char **NESTGPU_GetScalParamNames(int i_node);
int NESTGPU_GetNScalParam(int i_node);
char **NESTGPU_GetPortParamNames(int i_node);
int NESTGPU_GetNGroupParam(int i_node);
char **NESTGPU_GetGroupParamNames(int i_node);
int NESTGPU_GetNPortParam(int i_node);
char **NESTGPU_GetArrayParamNames(int i_node);
int NESTGPU_GetNArrayParam(int i_node);
char **NESTGPU_GetArrayVarNames(int i_node);
int NESTGPU_GetNArrayVar(int i_node);

/* connection queries: src/nestgpu_C.h:256-273 */
int *NESTGPU_GetSeqSeqConnections(int i_source, int n_source, int i_target, int n_target,
                                  int syn_group, int *n_conn);
int *NESTGPU_GetSeqGroupConnections(int i_source, int n_source, int *i_target, int n_target,
                                    int syn_group, int *n_conn);
int *NESTGPU_GetGroupSeqConnections(int *i_source, int n_source, int i_target, int n_target,
                                    int syn_group, int *n_conn);
int *NESTGPU_GetGroupGroupConnections(int *i_source, int n_source, int *i_target, int n_target,
                                      int syn_group, int *n_conn);
int NESTGPU_GetConnectionStatus(int i_source, int i_group, int i_conn, int *i_target,
                                unsigned char *port, unsigned char *syn_group, float *delay,
                                float *weight);

/* synapse groups: src/nestgpu_C.h:275-287.  Models "stdp" (tau_plus, tau_minus, lambda, alpha,
   mu_plus, mu_minus, Wmax; src/stdp.h:70-94) and "test_syn_model" (fact, offset); indices are
   1-based, 0 being the static synapse.  A network with plastic connections advances one time
   step per kernel batch (the weight changes of a step see that step's spikes). */
int NESTGPU_CreateSynGroup(char *model_name);
int NESTGPU_GetSynGroupNParam(int i_syn_group);
char **NESTGPU_GetSynGroupParamNames(int i_syn_group);
int NESTGPU_IsSynGroupParam(int i_syn_group, char *param_name);
int NESTGPU_GetSynGroupParamIdx(int i_syn_group, char *param_name);
float NESTGPU_GetSynGroupParam(int i_syn_group, char *param_name);
int NESTGPU_SetSynGroupParam(int i_syn_group, char *param_name, float val);

/* spike counting and spike-time recording: src/nestgpu_C.h:289-301 */
int NESTGPU_ActivateSpikeCount(int i_node, int n_node);
int NESTGPU_ActivateRecSpikeTimes(int i_node, int n_node, int max_n_rec_spike_times);
int NESTGPU_SetRecSpikeTimesStep(int i_node, int n_node, int rec_spike_times_step);
int NESTGPU_GetNRecSpikeTimes(int i_node);
int NESTGPU_GetRecSpikeTimes(int i_node, int n_node, int **n_spike_times_pt,
                             float ***spike_times_pt);

/* external neurons (not supported, error 2): src/nestgpu_C.h:303-307 */
int NESTGPU_PushSpikesToNodes(int n_spikes, int *node_id);
int NESTGPU_GetExtNeuronInputSpikes(int *n_spikes, int **node, int **port, float **spike_height,
                                    int include_zeros);

/* group parameters and kernel parameters: src/nestgpu_C.h:309-352 */
int NESTGPU_SetNeuronGroupParam(int i_node, int n_node, char *param_name, float val);
int NESTGPU_IsNeuronGroupParam(int i_node, char *param_name);
float NESTGPU_GetNeuronGroupParam(int i_node, char *param_name);
int NESTGPU_GetNBoolParam();
char **NESTGPU_GetBoolParamNames();
int NESTGPU_IsBoolParam(char *param_name);
int NESTGPU_GetBoolParamIdx(char *param_name);
bool NESTGPU_GetBoolParam(char *param_name);
int NESTGPU_SetBoolParam(char *param_name, bool val);
int NESTGPU_GetNFloatParam();
char **NESTGPU_GetFloatParamNames();
int NESTGPU_IsFloatParam(char *param_name);
int NESTGPU_GetFloatParamIdx(char *param_name);
float NESTGPU_GetFloatParam(char *param_name);
int NESTGPU_SetFloatParam(char *param_name, float val);
int NESTGPU_GetNIntParam();
char **NESTGPU_GetIntParamNames();
int NESTGPU_IsIntParam(char *param_name);
int NESTGPU_GetIntParamIdx(char *param_name);
int NESTGPU_GetIntParam(char *param_name);
int NESTGPU_SetIntParam(char *param_name, int val);
int NESTGPU_RemoteCreate(int i_host, char *model_name, int n_neuron, int n_port);

/* ---- engine extensions (no counterpart in the reference) ---- */

/* Release an array returned by a getter (the reference's Python front-end leaks them). */
void NGPU_FreeArray(void *p);

/* Destroy the engine instance so that the next call starts a new, empty network. */
int NGPU_Reset();

/* Counters since calibration: RK5 derivative evaluations, synaptic events delivered,
   spikes emitted; wall time of the last Simulate step loop [s]; steps run; device status bits
   (1 ring overflow, 2 RK5 iteration cap, 4 V_m/w guard reset, 8 spike-time buffer full). */
int NGPU_GetStats(unsigned long long *n_derivs, unsigned long long *n_events,
                  unsigned long long *n_spikes, double *sim_seconds, long long *steps,
                  unsigned int *status);

/* Bulk connection import: n edges with their own source, target, receptor, weight and
   delay (ms).  Same validation and storage as n single connections, without per-call cost. */
int NGPU_ConnectArrays(size_t n, int *source, int *target, unsigned char *port, float *weight,
                       float *delay);

/* Number of engine kernels launched since the engine was created (a CUDA-graph replay counts
   each kernel node it runs). */
long long NGPU_GetLaunchCount();

/* Device time [ms] of the last NESTGPU_Simulate call: CUDA events recorded on the engine's
   stream around its step loop and final input fold. */
double NGPU_GetSimDeviceMs();

/* Run n ordinary simulation steps with each kernel bracketed by CUDA events; writes the
   average device time per step [ms] of the neuron-update kernels, the record gather and the
   spike delivery into ms_out[0..2]; returns 3. */
int NGPU_ProfileSteps(int n, double *ms_out);

/* Fixed in-degree block generated on the device at calibration: each of the n_target
   targets draws `indegree` sources uniformly (with replacement) from the n_source nodes
   starting at i_source, with delays uniform on the time grid in [delay_min, delay_max] ms.
   Unlike NESTGPU's fixed_indegree rule (one draw shared by all targets of a call), every
   target draws its own sources.  The edges live only on the device (GetConnections does not
   list them).  Edge kk of the block's t-th target draws one Philox4x32-10 block keyed by
   `seed` with counter (t, kk, 0, 0x9E3779B9): source i_source + floor(x * n_source / 2^32),
   delay step round(delay_min/dt) - 1 + floor(y * n_steps / 2^32).  The draws depend only on
   the block's own indices and seed, so blocks meant to differ need different seeds. */
int NGPU_ConnectFixedIndegreeGPU(int i_source, int n_source, int i_target, int n_target, int indegree,
                                 int port, float weight, float delay_min, float delay_max,
                                 unsigned long long seed);

/* Connect calls with the fixed_total_number, fixed_indegree or fixed_outdegree rule, static
   synapses and at least n edges (default 65536) keep their random numbers (the same cuRAND
   draws as otherwise), weights and delays on the device; their edges are expanded into the
   delivery layout on the device at calibration and reach the host connection store only when
   a connection query needs them.  Needs a GPU; results and GetConnections do not depend on
   it.  No counterpart in the reference (src/connect_rules.h:161-338 expands on the host). */
int NGPU_SetDeviceRuleMinEdges(long long n);

/* poisson_generator nodes i_node .. i_node+n_node-1 draw from Poisson streams stream ..
   stream+n_node-1 (before calibration).  A generator's draw for its j-th out-edge (in
   connection order) at time index t depends only on (kernel seed, stream, j, t); by default
   the stream is the generator's index among all poisson_generator nodes.  Giving each
   generator of an independent sub-network its own fixed stream makes that sub-network's
   input the same wherever it sits in a larger network.  No counterpart in the reference
   (its generators draw from per-edge cuRAND states). */
int NGPU_SetPoissonStream(int i_node, int n_node, unsigned int stream);

/* Shape of the recurrent delivery layout after calibration: the number of nodes, the smallest
   delay step (round(delay/dt) - 1) and the number of delay steps spanned, and the number of
   edges.  No counterpart in the reference (its layout is the per-source connection groups of
   src/connect.h:58-70). */
int NGPU_GetDeliveryShape(int *n_nodes, int *dmin, int *dspan, long long *n_edges);

/* Copy the recurrent delivery layout to host arrays: seg_off[n_nodes*dspan + 1] (segment
   (source s, delay step dmin + d) holds edges seg_off[s*dspan + d] .. seg_off[s*dspan + d + 1]
   - 1), and per edge its target node, receptor port and weight (any of the three may be
   NULL).  The order inside a segment is unspecified. */
int NGPU_GetDeliveryCsr(long long *seg_off, int *target, unsigned char *port, float *weight);

/* Thread blocks of the spike-delivery kernel (0 = chosen from the number of nodes with
   outgoing connections, at most 8 per SM).  Results do not depend on it. */
int NGPU_SetDeliverBlocks(int n);

/* Upper bound of the number of time steps integrated per batch (default 32, before
   calibration).  A batch never exceeds the minimum connection delay in steps, so spikes
   emitted inside it cannot reach a target inside it; 1 advances step by step.  Results do
   not depend on it. */
int NGPU_SetBatchMax(int n);

/* RK5 steps a neuron may take in the main update kernel per batch beyond one per time step
   before it is handed to the straggler kernel (default 4; 0 = no hand-off).  Results do not
   depend on it. */
int NGPU_SetRk5Budget(int n);

/* Pack a device-resident edge list into the spike-delivery layout: edges grouped into
   segments by (source node, delay index).  All pointers are device pointers.
     src[n]     source node of each edge, 0 <= src < n_nodes
     dly[n]     delay index relative to the smallest delay, 0 <= dly < dspan
     target[n]  accumulator index of each edge (receptor row offset + target)
     weight[n]  weight
   Writes seg_off[n_nodes*dspan + 1] (start of each segment; seg_off[last] = n) and edge[n]
   (8-byte records {uint32 target, float weight}; order inside a segment unspecified).
   Scratch (per-segment counters, scan workspace) comes from cudaMalloc and is released
   before returning.  stream: a cudaStream_t or NULL.  Returns 0, or -1 with the error set
   (code 255 for an out-of-range source or delay index). */
int NGPU_BuildDeliveryCsr(const int *src, const int *dly, const unsigned *target, const float *weight,
                          size_t n, int n_nodes, int dspan, unsigned long long *seg_off, void *edge,
                          void *stream);

/* NGPU_BuildDeliveryCsr for callers that cannot allocate device memory.  No counterpart in
   the reference.  A process whose device heap belongs to another allocator (a PyTorch
   program) or that divides each GPU into fixed pools at start-up may not call cudaMalloc;
   this variant takes its scratch from a static device array of about 4.3 MiB that every GPU
   loading the library holds until exit.  Same arguments and results as
   NGPU_BuildDeliveryCsr; n_nodes * dspan must not exceed 524288 segments (larger problems
   are rejected with error code 2).  All calls share the array: calls that overlap on the
   GPU race.  Each call is synchronous: it returns after its work on `stream` has finished
   and its status word (an out-of-range source or delay index, code 255) has been read
   back.  The first call on a device looks up the array's device address, with that device
   current; make it before any stream capture. */
int NGPU_BuildDeliveryCsrNoAlloc(const int *src, const int *dly, const unsigned *target,
                                 const float *weight, size_t n, int n_nodes, int dspan,
                                 unsigned long long *seg_off, void *edge, void *stream);

/* Steps captured per CUDA graph (default 100). */
int NGPU_SetGraphSteps(int n);
/* Steps per time batch of the calibrated network: the kernels advance this many steps per
   launch (the minimum delay in steps + 1, at most 32 and at most the batch_max setting). */
int NGPU_GetBatchLength(void);

/* Threads per block of the aeif update kernel (64, 128 or 256; default 128). */
int NGPU_SetUpdateThreads(int n);
/* 1: use the register-capped variant of the aeif update kernel (three 256-thread blocks per
   SM, more warps in flight, a few register spills); 2: with the trial-per-iteration update
   and uniform parameters, a variant capped at five 128-thread blocks per SM (96 registers,
   blocks of at most 128 threads); 0: the unconstrained one (default). */
int NGPU_SetUpdateOccupancy(int on);
/* 1: the aeif update kernel advances one RK5 trial per loop iteration (a rejected trial is
   retried in the next iteration beside the neighbouring lanes' next trials); 0: one whole
   step, rejected trials included, per iteration (default).  Results do not depend on it. */
int NGPU_SetUpdateTrialIter(int on);
/* 1: with 32-lane delivery work items, lanes whose edges share a target add their products
   and one lane issues the reduction (warp-aggregated reductions); 0: one reduction per edge
   (default).  Results do not depend on it. */
int NGPU_SetDeliverAggregate(int on);
/* 1: each delivery work group loads its next work item's spike and segment offsets before it
   streams the current segment (a two-stage software pipeline); 0: one item after the other.
   Results do not depend on it. */
int NGPU_SetDeliverPrefetch(int on);
/* 1: in a network whose neurons are all iaf_psc_exp (Poisson generators aside), with no
   plastic connections and one process, each spike's out-edges are added to the target
   accumulators by the update kernel's block in the step the spike is emitted, into a ring of
   accumulator slots indexed by arrival step, and no delivery kernel runs; 0 (default): the
   delivery kernel.  Takes effect at calibration (call it before the first Simulate); results do not
   depend on it, except that the event counter (NGPU_GetStats) then counts a spike's edges when it
   is emitted, not when they arrive.  Replaces the delivery path of src/nestgpu.cu:469-635 (SendSpike, then
   CollectSpikeKernel in the next step); no reference counterpart as a switch. */
int NGPU_SetDeliverPush(int on);
/* 1 if delivery at emission is active (after calibration), else 0. */
int NGPU_DeliverPushActive(void);
/* Lanes per spike-delivery work item (8, 16 or 32; default 32): one item is the out-edge
   segment of one (source, delay) pair; short segments leave fewer lanes idle with small
   groups. */
int NGPU_SetDeliverGroup(int g);
/* 1: a network whose neurons are all iaf_psc_exp runs its steps in one cooperative launch per
   CUDA-graph's worth of steps (delivery and update separated by grid barriers with bounded
   waits); 0 (default): per-batch launches in CUDA graphs.  Results are the same either way; the
   autotuner tries both. */
int NGPU_SetPersistent(int on);
/* 1: the kernels of a time batch are launched with programmatic stream serialization, so each
   kernel's launch and block scheduling overlap the end of the kernel before it (every such
   kernel first waits for its predecessor's completion and memory, so results are the same);
   used where the batch is one chain of kernels on one stream (not with plastic synapses or
   with aeif and other spiking groups together).  0: plain stream order.  A negative value
   (default) uses it for batches of one time step only (a minimum delay of one step), where a
   step is two short launches.  The autotuner tries both.  No counterpart in the reference. */
int NGPU_SetProgrammaticLaunch(int on);
/* Test hook for the failure path of the persistent loop: with extra > 0 its grid barriers wait
   for more blocks than the launch has, so each wait runs out after its bounded number of polls
   (a second or two); the kernel records the timeout and returns, and the Simulate call fails
   with error code 2 while the GPU context stays usable.  0 (default) disables it. */
int NGPU_TestBarrierTimeout(int extra);
/* Test hook for the failure path of the step-model training kernel: with on != 0 its
   tensor-core products are issued but their completion is never signalled on the block's
   mbarrier, so the bounded wait runs out; the kernel records it, releases its tensor memory
   and returns, and NGPU_MlpGrad / NGPU_StepModelTrain fail with error code 2 while the GPU
   context stays usable.  0 (default) disables it.  No counterpart in the reference. */
int NGPU_TestTensorWaitTimeout(int on);
/* Autotuner of the launch mappings (no counterpart in the reference): on the calibrated
   network, after 4 x `steps` warm-up steps, times `steps` simulation steps per candidate of the
   update block size, the update kernel variant, the delivery lane group, the delivery grid and
   the RK5 step budget, each candidate twice (forward and reverse order), in a coordinate
   descent of two passes, and keeps the fastest.  The trials are ordinary simulation steps, so
   the network advances by them.  Returns the number of trials (-1 on error) and the chosen
   values. */
int NGPU_Autotune(int steps, int *update_threads, int *deliver_group, int *deliver_blocks,
                  int *rk5_budget);
/* The current launch mapping: writes min(n, 10) of {update block size, register-capped update
   variant, delivery lane group, delivery grid (0: automatic), RK5 step budget, persistent loop,
   programmatic launch, trial-per-iteration update, warp-aggregated delivery, pipelined delivery}
   and returns 10 (-1 on error).  No counterpart in the reference. */
int NGPU_GetLaunchMapping(int *vals, int n);
/* Measured rate (1e9 per second) of FP64 reductions to uniformly random addresses of a
   `bytes`-byte device buffer, `n_ops` in total: the access pattern of the spike delivery's
   accumulator updates, used as that kernel's roofline denominator.  -1 on error.  No
   counterpart in the reference. */
double NGPU_MeasureReductionRate(size_t bytes, long long n_ops);

/* 1: draw connection random numbers with cuRAND's host generator instead of the device
   generator the reference uses (integer streams are identical, normal streams are not);
   lets a CPU checker reproduce normal-distributed weights and delays exactly. */
int NGPU_SetHostRng(int on);

/* ---- Learned RK5 step-size proposal.  No counterpart in the reference: the reference's
   only step-size rule is the controller of src/rk5.h:134-150, which stays in place here.
   Features of a step (after its first derivative evaluation): V_m, w, the first state
   variable of ports 0..3, dV_m/dt, the sum of that variable's derivatives over all
   ports, log of the controller's h, log of the remaining interval.  Network 10-32-32-1
   (ReLU), BF16 weights, FP32 accumulation; proposal = safety * exp(out * label_sigma +
   label_mu), raised to at least floor * (the controller's h) when floor > 0.  Flat
   parameter vector (NGPU_StepModelNParams() = 1465 floats): mu[10], inv_sigma[10],
   W1[32][10], b1[32], W2[32][32], b2[32], W3[32], b3, label_mu, label_sigma, safety,
   floor.  All return 0 (count functions: the count) or -1 on error. */
int NGPU_StepModelNParams(void);
/* Log one tuple of 12 floats (10 features, accepted h, error of the accepted trial) per
   accepted RK5 step of every aeif neuron in the following Simulate calls; at most
   `capacity` tuples are kept. */
int NGPU_Rk5LogStart(long long capacity);
int NGPU_Rk5LogStop(void);
long long NGPU_Rk5LogCount(long long *offered);
int NGPU_Rk5LogGet(float *out, long long first, long long n);
/* Train the network on the logged tuples (steps whose controller h would not reach the end
   of the time step) with the engine's GPU kernels: feature / target normalisation,
   minibatch Adam on the mean squared error of the target log(h * err^-0.2); the result
   becomes the engine's model. */
int NGPU_StepModelTrain(long long iters, int batch, float lr, float safety, float floor,
                        unsigned long long seed, long long *n_used, float *final_loss);
int NGPU_StepModelSet(const float *params);
int NGPU_StepModelGet(float *params);
/* 1: the network proposes the first trial h of every RK5 step whose controller h would not
   reach the end of the time step; the error test, the rejection shrink and the controller
   update are unchanged, and invalid proposals fall back to the controller's h. */
int NGPU_StepModelEnable(int on);
/* 1: analysis mode for the learned proposal's ceiling: every RK5 step of the aeif groups
   (1 to 4 receptor ports) starts from the largest step size that passes the unchanged error
   test (a bisection whose trials are not counted), so the evaluation counter shows the floor
   no step-size proposal can go below; 0: back to the plain controller.  No counterpart in the
   reference. */
int NGPU_StepBoundMode(int on);
/* Network output for n feature rows, and the mean squared error with its gradient over the
   trainable block W1..b3 (1441 floats), computed by the GPU kernels on host buffers (the
   gradient by the training kernel: tensor-core products of BF16 operands, FP32 sums). */
int NGPU_MlpForward(const float *params, const float *feat, int n, float *out);
int NGPU_MlpGrad(const float *params, const float *feat, const float *target, int n, float *grad,
                 float *loss);

#ifdef __cplusplus
}
#endif

#endif
