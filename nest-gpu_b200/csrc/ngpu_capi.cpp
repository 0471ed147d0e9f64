// extern "C" entry points of libnestgpu_b200.so (declared in include/nestgpu_b200.h).
// Error convention of the reference (src/propagate_error.h:4-30): clear the error
// state, run, map an engine error to code 2, bad_alloc to 1, anything else to 255;
// exit with that code unless SetOnException(1) asked to return to the caller.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/nestgpu_b200.h"
#include "ngpu_engine.h"

using namespace ngpu;

namespace {

struct ErrState {
  bool flag = false;
  std::string message;
  unsigned char code = 0;
  int on_exception = 0;   // 0: exit (reference default for C callers), 1: return
};
thread_local ErrState g_err;

// connection / synapse specification staged by the Set*Spec* calls (src/nestgpu_C.cpp:39-40)
struct ConnSpecC {
  int rule = 1;   // all_to_all
  int total_num = 0, indegree = 0, outdegree = 0;
};
struct SynSpecC {
  int syn_group = 0, port = 0;
  float weight = 0.0f, delay = 0.0f;
  float *weight_array = nullptr, *delay_array = nullptr;
};
thread_local ConnSpecC g_conn;
thread_local SynSpecC g_syn;
thread_local double g_last_device_ms = 0.0;

void fail(unsigned char code, const std::string &msg) {
  g_err.flag = true;
  g_err.code = code;
  g_err.message = msg;
  if (g_err.on_exception == 0) {
    std::fprintf(stderr, "%s\n", msg.c_str());
    std::exit(code);
  }
}

template <class F> auto guard(F f, decltype(f()) on_err) -> decltype(f()) {
  g_err.flag = false;
  g_err.code = 0;
  g_err.message.clear();
  try {
    return f();
  } catch (NgpuError &e) {
    fail(2, e.what());
  } catch (std::bad_alloc &) {
    fail(1, "Memory allocation error");
  } catch (std::exception &e) {
    fail(255, e.what());
  } catch (...) {
    fail(255, "Unknown error");
  }
  return on_err;
}

std::vector<int> seq(int i0, int n) {
  std::vector<int> v(n > 0 ? n : 0);
  for (int i = 0; i < n; i++) v[i] = i0 + i;
  return v;
}
std::vector<int> lst(const int *a, int n) { return std::vector<int>(a, a + (n > 0 ? n : 0)); }

template <class T> T *malloc_copy(const std::vector<T> &v) {
  T *p = (T *)std::malloc(std::max<size_t>(v.size(), 1) * sizeof(T));
  if (!p) throw std::bad_alloc();
  if (!v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
  return p;
}

char **name_list(const std::vector<std::string> &names) {
  char **a = (char **)std::malloc(std::max<size_t>(names.size(), 1) * sizeof(char *));
  for (size_t i = 0; i < names.size(); i++) {
    a[i] = (char *)std::malloc(names[i].size() + 1);
    std::strcpy(a[i], names[i].c_str());
  }
  return a;
}

const char *kFloatParam[] = {"time_resolution", "max_spike_num_fact", "max_spike_per_host_fact"};
const char *kIntParam[] = {"rnd_seed", "verbosity_level", "max_spike_buffer_size", "remote_spike_height_flag"};
const char *kBoolParam[] = {"print_time"};

int idx_of(const char *const *names, int n, const char *name) {
  for (int i = 0; i < n; i++)
    if (std::strcmp(names[i], name) == 0) return i;
  return -1;
}

Engine &E() { return engine(); }

int do_connect(const int *src, int s0, int ns, const int *tgt, int t0, int nt) {
  int degree = 0;
  switch (g_conn.rule) {
  case 2: degree = g_conn.total_num; break;
  case 3: degree = g_conn.indegree; break;
  case 4: degree = g_conn.outdegree; break;
  default: break;
  }
  E().connect_rule(g_conn.rule, src, s0, ns, tgt, t0, nt, degree, g_syn.port, g_syn.syn_group,
                   g_syn.weight, g_syn.delay, g_syn.weight_array, g_syn.delay_array);
  return 0;
}

}  // namespace

extern "C" {

char *NESTGPU_GetErrorMessage() { return (char *)g_err.message.c_str(); }
unsigned char NESTGPU_GetErrorCode() { return g_err.code; }
void NESTGPU_SetOnException(int on_exception) { g_err.on_exception = on_exception; }

int NESTGPU_SetRandomSeed(unsigned long long seed) {
  return guard([&] { E().set_seed(seed); return 0; }, 0);
}
int NESTGPU_SetTimeResolution(float t) {
  return guard([&] { E().set_time_resolution(t); return 0; }, 0);
}
float NESTGPU_GetTimeResolution() { return guard([&] { return E().dt; }, 0.0f); }
int NESTGPU_SetMaxSpikeBufferSize(int n) {
  return guard([&] { E().max_spike_buffer_size = n; return 0; }, 0);
}
int NESTGPU_GetMaxSpikeBufferSize() { return guard([&] { return E().max_spike_buffer_size; }, 0); }
int NESTGPU_SetSimTime(float t) { return guard([&] { E().sim_time = t; return 0; }, 0); }
int NESTGPU_SetVerbosityLevel(int v) { return guard([&] { E().verbosity = v; return 0; }, 0); }

int NESTGPU_Create(char *model_name, int n, int n_port) {
  return guard([&] { return E().create(model_name, n, n_port); }, 0);
}
int NESTGPU_CreatePoissonGenerator(int n, float rate) {
  return guard([&] { return E().create_poisson_generator(n, rate); }, 0);
}
int NESTGPU_CreateRecord(char *file_name, char *var_name_arr[], int *i_node_arr, int *port_arr,
                         int n_node) {
  return guard([&] {
    std::vector<std::string> vars;
    for (int i = 0; i < n_node; i++) vars.push_back(var_name_arr[i]);
    return E().create_record(file_name ? file_name : "", vars, lst(i_node_arr, n_node),
                             lst(port_arr, n_node));
  }, 0);
}
int NESTGPU_GetRecordDataRows(int i) { return guard([&] { return (int)E().record(i).data.size(); }, 0); }
int NESTGPU_GetRecordDataColumns(int i) {
  return guard([&] { return (int)E().record(i).var.size() + 1; }, 0);
}
float **NESTGPU_GetRecordData(int i) {
  return guard([&] {
    RecordSpec &r = E().record(i);
    r.row_ptr.resize(r.data.size());
    for (size_t k = 0; k < r.data.size(); k++) r.row_ptr[k] = r.data[k].data();
    return r.row_ptr.data();
  }, (float **)nullptr);
}

// ---- parameters and variables
int NESTGPU_SetNeuronScalParam(int i_node, int n, char *name, float val) {
  return guard([&] { E().set_scalar(seq(i_node, n), name, val); return 0; }, 0);
}
int NESTGPU_SetNeuronArrayParam(int i_node, int n, char *name, float *p, int sz) {
  return guard([&] { E().set_port_or_array(seq(i_node, n), name, p, sz); return 0; }, 0);
}
int NESTGPU_SetNeuronPtScalParam(int *i_node, int n, char *name, float val) {
  return guard([&] {
    for (int i = 0; i < n; i++) E().set_scalar({i_node[i]}, name, val);
    return 0;
  }, 0);
}
int NESTGPU_SetNeuronPtArrayParam(int *i_node, int n, char *name, float *p, int sz) {
  return guard([&] {
    for (int i = 0; i < n; i++) E().set_port_or_array({i_node[i]}, name, p, sz);
    return 0;
  }, 0);
}
int NESTGPU_IsNeuronScalParam(int i_node, char *name) {
  return guard([&] { return (int)(E().locate(i_node, name) == K_SCAL_PARAM); }, 0);
}
int NESTGPU_IsNeuronPortParam(int i_node, char *name) {
  return guard([&] { return (int)(E().locate(i_node, name) == K_PORT_PARAM); }, 0);
}
int NESTGPU_IsNeuronArrayParam(int i_node, char *name) {
  return guard([&] { return (int)(E().locate(i_node, name) == K_ARRAY_PARAM); }, 0);
}
int NESTGPU_SetNeuronIntVar(int i_node, int n, char *name, int val) {
  return guard([&] { E().set_int_var(seq(i_node, n), name, val); return 0; }, 0);
}
int NESTGPU_SetNeuronScalVar(int i_node, int n, char *name, float val) {
  return guard([&] { E().set_scalar(seq(i_node, n), name, val); return 0; }, 0);
}
int NESTGPU_SetNeuronArrayVar(int i_node, int n, char *name, float *v, int sz) {
  return guard([&] { E().set_port_or_array(seq(i_node, n), name, v, sz); return 0; }, 0);
}
int NESTGPU_SetNeuronPtIntVar(int *i_node, int n, char *name, int val) {
  return guard([&] {
    for (int i = 0; i < n; i++) E().set_int_var({i_node[i]}, name, val);
    return 0;
  }, 0);
}
int NESTGPU_SetNeuronPtScalVar(int *i_node, int n, char *name, float val) {
  return guard([&] {
    for (int i = 0; i < n; i++) E().set_scalar({i_node[i]}, name, val);
    return 0;
  }, 0);
}
int NESTGPU_SetNeuronPtArrayVar(int *i_node, int n, char *name, float *v, int sz) {
  return guard([&] {
    for (int i = 0; i < n; i++) E().set_port_or_array({i_node[i]}, name, v, sz);
    return 0;
  }, 0);
}
int NESTGPU_IsNeuronIntVar(int i_node, char *name) {
  return guard([&] { return (int)(E().locate(i_node, name) == K_INT_VAR); }, 0);
}
int NESTGPU_IsNeuronScalVar(int i_node, char *name) {
  return guard([&] { return (int)(E().locate(i_node, name) == K_SCAL_VAR); }, 0);
}
int NESTGPU_IsNeuronPortVar(int i_node, char *name) {
  return guard([&] { return (int)(E().locate(i_node, name) == K_PORT_VAR); }, 0);
}
int NESTGPU_IsNeuronArrayVar(int i_node, char *name) {
  (void)i_node;
  (void)name;
  return guard([&] { return 0; }, 0);   // no model on this path has array variables
}
int NESTGPU_GetNeuronParamSize(int i_node, char *name) {
  return guard([&] { return E().param_size(i_node, name); }, 0);
}
int NESTGPU_GetNeuronVarSize(int i_node, char *name) {
  return guard([&] { return E().var_size(i_node, name); }, 0);
}
float *NESTGPU_GetNeuronParam(int i_node, int n, char *name) {
  return guard([&] { return malloc_copy(E().get_values(seq(i_node, n), name)); }, (float *)nullptr);
}
float *NESTGPU_GetNeuronPtParam(int *i_node, int n, char *name) {
  return guard([&] {
    std::vector<float> out;
    for (int i = 0; i < n; i++) {
      auto v = E().get_values({i_node[i]}, name);
      out.insert(out.end(), v.begin(), v.end());
    }
    return malloc_copy(out);
  }, (float *)nullptr);
}
float *NESTGPU_GetArrayParam(int i_node, char *name) {
  return guard([&] { return malloc_copy(E().get_array_param(i_node, name)); }, (float *)nullptr);
}
int *NESTGPU_GetNeuronIntVar(int i_node, int n, char *name) {
  return guard([&] {
    int *p = (int *)std::malloc(std::max<size_t>(n > 0 ? (size_t)n : 0, 1) * sizeof(int));
    if (!p) throw std::bad_alloc();
    try {
      E().get_int_values_seq(i_node, n, name, p);
    } catch (...) {
      std::free(p);
      throw;
    }
    return p;
  }, (int *)nullptr);
}
int *NESTGPU_GetNeuronPtIntVar(int *i_node, int n, char *name) {
  return guard([&] {
    std::vector<int> out;
    for (int i = 0; i < n; i++) out.push_back(E().get_int_values({i_node[i]}, name)[0]);
    return malloc_copy(out);
  }, (int *)nullptr);
}
float *NESTGPU_GetNeuronVar(int i_node, int n, char *name) {
  return guard([&] { return malloc_copy(E().get_values(seq(i_node, n), name)); }, (float *)nullptr);
}
float *NESTGPU_GetNeuronPtVar(int *i_node, int n, char *name) {
  return NESTGPU_GetNeuronPtParam(i_node, n, name);
}
float *NESTGPU_GetArrayVar(int i_node, char *name) {
  return guard([&]() -> float * {
    (void)i_node;
    throw NgpuError(std::string("Unrecognized array variable ") + name);
  }, (float *)nullptr);
}

// ---- simulation
int NESTGPU_Calibrate() { return guard([&] { E().calibrate(); return 0; }, 0); }
int NESTGPU_Simulate() { return guard([&] { E().simulate(E().sim_time); return 0; }, 0); }
int NESTGPU_StartSimulation() { return guard([&] { E().start_simulation(); return 0; }, 0); }
int NESTGPU_SimulationStep() { return guard([&] { E().simulation_step(); return 0; }, 0); }
int NESTGPU_EndSimulation() { return guard([&] { E().end_simulation(); return 0; }, 0); }

// ---- MPI: one process
int NESTGPU_ConnectMpiInit(int, char *[]) {
  return guard([&]() -> int { throw NgpuError("MPI is not available in this engine (single GPU)"); }, 0);
}
int NESTGPU_MpiId() { return 0; }
int NESTGPU_MpiNp() { return 1; }
int NESTGPU_ProcMaster() { return 1; }
int NESTGPU_MpiFinalize() { return 0; }

// ---- random numbers
unsigned int *NESTGPU_RandomInt(size_t n) {
  return guard([&] { return malloc_copy(E().random_int(n)); }, (unsigned *)nullptr);
}
float *NESTGPU_RandomUniform(size_t n) {
  return guard([&] { return malloc_copy(E().random_uniform(n)); }, (float *)nullptr);
}
float *NESTGPU_RandomNormal(size_t n, float mean, float sd) {
  return guard([&] { return malloc_copy(E().random_normal(n, mean, sd)); }, (float *)nullptr);
}
float *NESTGPU_RandomNormalClipped(size_t n, float mean, float sd, float vmin, float vmax, float vstep) {
  return guard([&] { return malloc_copy(E().random_normal_clipped(n, mean, sd, vmin, vmax, vstep)); },
               (float *)nullptr);
}

// ---- connections
int NESTGPU_Connect(int src, int tgt, unsigned char port, unsigned char syn_group, float w, float d) {
  return guard([&] { E().connect1(src, tgt, port, syn_group, w, d); return 0; }, 0);
}
int NESTGPU_ConnSpecInit() { return guard([&] { g_conn = ConnSpecC(); return 0; }, 0); }
int NESTGPU_SetConnSpecParam(char *name, int value) {
  return guard([&] {
    std::string s(name);
    if (s == "rule") {
      if (value < 0 || value > 4) throw NgpuError("Unknown connection rule");
      g_conn.rule = value;
    } else if (s == "indegree") {
      if (value < 0) throw NgpuError("Indegree must be >=0");
      g_conn.indegree = value;
    } else if (s == "outdegree") {
      if (value < 0) throw NgpuError("Outdegree must be >=0");
      g_conn.outdegree = value;
    } else if (s == "total_num") {
      if (value < 0) throw NgpuError("total_num must be >=0");
      g_conn.total_num = value;
    } else {
      throw NgpuError("Unknown connection int parameter");
    }
    return 0;
  }, 0);
}
int NESTGPU_ConnSpecIsParam(char *name) {
  std::string s(name);
  return guard([&] { return (int)(s == "rule" || s == "indegree" || s == "outdegree" || s == "total_num"); }, 0);
}
int NESTGPU_SynSpecInit() { return guard([&] { g_syn = SynSpecC(); return 0; }, 0); }
int NESTGPU_SetSynSpecIntParam(char *name, int value) {
  return guard([&] {
    std::string s(name);
    if (s == "synapse_group") {
      if (value < 0) throw NgpuError("Unknown synapse group");
      g_syn.syn_group = value;
    } else if (s == "receptor") {
      if (value < 0) throw NgpuError("Port index must be >=0");
      g_syn.port = value;
    } else {
      throw NgpuError("Unknown synapse int parameter");
    }
    return 0;
  }, 0);
}
int NESTGPU_SetSynSpecFloatParam(char *name, float value) {
  return guard([&] {
    std::string s(name);
    if (s == "weight") g_syn.weight = value;
    else if (s == "delay") {
      if (value < 0) throw NgpuError("Delay must be >=0");
      g_syn.delay = value;
    } else throw NgpuError("Unknown synapse float parameter");
    return 0;
  }, 0);
}
int NESTGPU_SetSynSpecFloatPtParam(char *name, float *arr) {
  return guard([&] {
    std::string s(name);
    if (s == "weight_array") g_syn.weight_array = arr;
    else if (s == "delay_array") g_syn.delay_array = arr;
    else throw NgpuError("Unknown synapse array parameter");
    return 0;
  }, 0);
}
int NESTGPU_SynSpecIsIntParam(char *name) {
  std::string s(name);
  return guard([&] { return (int)(s == "synapse_group" || s == "receptor"); }, 0);
}
int NESTGPU_SynSpecIsFloatParam(char *name) {
  std::string s(name);
  return guard([&] { return (int)(s == "weight" || s == "delay"); }, 0);
}
int NESTGPU_SynSpecIsFloatPtParam(char *name) {
  std::string s(name);
  return guard([&] { return (int)(s == "weight_array" || s == "delay_array"); }, 0);
}
int NESTGPU_ConnectSeqSeq(int i_source, int n_source, int i_target, int n_target) {
  return guard([&] { return do_connect(nullptr, i_source, n_source, nullptr, i_target, n_target); }, 0);
}
int NESTGPU_ConnectSeqGroup(int i_source, int n_source, int *i_target, int n_target) {
  return guard([&] { return do_connect(nullptr, i_source, n_source, i_target, 0, n_target); }, 0);
}
int NESTGPU_ConnectGroupSeq(int *i_source, int n_source, int i_target, int n_target) {
  return guard([&] { return do_connect(i_source, 0, n_source, nullptr, i_target, n_target); }, 0);
}
int NESTGPU_ConnectGroupGroup(int *i_source, int n_source, int *i_target, int n_target) {
  return guard([&] { return do_connect(i_source, 0, n_source, i_target, 0, n_target); }, 0);
}
static int no_mpi() {
  return guard([&]() -> int { throw NgpuError("MPI is not available in this engine (single GPU)"); }, 0);
}
int NESTGPU_RemoteConnectSeqSeq(int, int, int, int, int, int) { return no_mpi(); }
int NESTGPU_RemoteConnectSeqGroup(int, int, int, int, int *, int) { return no_mpi(); }
int NESTGPU_RemoteConnectGroupSeq(int, int *, int, int, int, int) { return no_mpi(); }
int NESTGPU_RemoteConnectGroupGroup(int, int *, int, int, int *, int) { return no_mpi(); }
int NESTGPU_RemoteCreate(int, char *, int, int) { return no_mpi(); }

// ---- names
#define NAMES(fn, kind)                                                                    \
  char **NESTGPU_Get##fn##Names(int i_node) {                                              \
    return guard([&] { return name_list(E().names(i_node, kind)); }, (char **)nullptr);     \
  }                                                                                        \
  int NESTGPU_GetN##fn(int i_node) {                                                       \
    return guard([&] { return (int)E().names(i_node, kind).size(); }, 0);                  \
  }
NAMES(IntVar, K_INT_VAR)
NAMES(ScalVar, K_SCAL_VAR)
NAMES(PortVar, K_PORT_VAR)
NAMES(ScalParam, K_SCAL_PARAM)
NAMES(PortParam, K_PORT_PARAM)
NAMES(GroupParam, K_GROUP_PARAM)
NAMES(ArrayParam, K_ARRAY_PARAM)
#undef NAMES
char **NESTGPU_GetArrayVarNames(int i_node) {
  return guard([&] { E().group_of(i_node); return name_list({}); }, (char **)nullptr);
}
int NESTGPU_GetNArrayVar(int i_node) { return guard([&] { E().group_of(i_node); return 0; }, 0); }

// ---- connection queries (n <= 0 for a sequence means every node)
static int *conn_ids(const int *src, int s0, int ns, const int *tgt, int t0, int nt, int syn_group,
                     int *n_conn) {
  const int N = E().n_nodes();
  if (!src && ns <= 0) { s0 = 0; ns = N; }
  if (!tgt && nt <= 0) { t0 = 0; nt = N; }
  std::vector<int> ids = E().get_connections(src, s0, ns, tgt, t0, nt, syn_group);
  *n_conn = (int)(ids.size() / 3);
  return malloc_copy(ids);
}
int *NESTGPU_GetSeqSeqConnections(int i_source, int n_source, int i_target, int n_target, int syn_group,
                                  int *n_conn) {
  return guard([&] { return conn_ids(nullptr, i_source, n_source, nullptr, i_target, n_target, syn_group, n_conn); },
               (int *)nullptr);
}
int *NESTGPU_GetSeqGroupConnections(int i_source, int n_source, int *i_target, int n_target, int syn_group,
                                    int *n_conn) {
  return guard([&] { return conn_ids(nullptr, i_source, n_source, i_target, 0, n_target, syn_group, n_conn); },
               (int *)nullptr);
}
int *NESTGPU_GetGroupSeqConnections(int *i_source, int n_source, int i_target, int n_target, int syn_group,
                                    int *n_conn) {
  return guard([&] { return conn_ids(i_source, 0, n_source, nullptr, i_target, n_target, syn_group, n_conn); },
               (int *)nullptr);
}
int *NESTGPU_GetGroupGroupConnections(int *i_source, int n_source, int *i_target, int n_target, int syn_group,
                                      int *n_conn) {
  return guard([&] { return conn_ids(i_source, 0, n_source, i_target, 0, n_target, syn_group, n_conn); },
               (int *)nullptr);
}
int NESTGPU_GetConnectionStatus(int i_source, int i_group, int i_conn, int *i_target,
                                unsigned char *port, unsigned char *syn_group, float *delay,
                                float *weight) {
  return guard([&] {
    E().connection_status(i_source, i_group, i_conn, i_target, port, syn_group, delay, weight);
    return 0;
  }, 0);
}

// ---- synapse groups (src/nestgpu_C.cpp:874-960, src/syn_model.cu:136-238)
int NESTGPU_CreateSynGroup(char *model_name) {
  return guard([&] { return E().create_syn_group(model_name); }, 0);
}
int NESTGPU_GetSynGroupNParam(int g) {
  return guard([&] { return (int)E().syn_group_param_names(g).size(); }, 0);
}
char **NESTGPU_GetSynGroupParamNames(int g) {
  return guard([&] { return name_list(E().syn_group_param_names(g)); }, (char **)nullptr);
}
int NESTGPU_IsSynGroupParam(int g, char *name) {
  return guard([&] {
    const std::vector<std::string> names = E().syn_group_param_names(g);
    return std::find(names.begin(), names.end(), std::string(name)) != names.end() ? 1 : 0;
  }, 0);
}
int NESTGPU_GetSynGroupParamIdx(int g, char *name) {
  return guard([&] { return E().syn_group_param_idx(g, name); }, 0);
}
float NESTGPU_GetSynGroupParam(int g, char *name) {
  return guard([&] { return E().get_syn_group_param(g, name); }, 0.0f);
}
int NESTGPU_SetSynGroupParam(int g, char *name, float val) {
  return guard([&] { E().set_syn_group_param(g, name, val); return 0; }, 0);
}

// ---- spike counting and recording
int NESTGPU_ActivateSpikeCount(int i_node, int n) {
  return guard([&] { E().activate_spike_count(i_node, n); return 0; }, 0);
}
int NESTGPU_ActivateRecSpikeTimes(int i_node, int n, int max_n) {
  return guard([&] { E().activate_rec_spike_times(i_node, n, max_n); return 0; }, 0);
}
int NESTGPU_SetRecSpikeTimesStep(int i_node, int n, int step) {
  return guard([&] { E().set_rec_spike_times_step(i_node, n, step); return 0; }, 0);
}
int NESTGPU_GetNRecSpikeTimes(int i_node) { return guard([&] { return E().n_rec_spike_times(i_node); }, 0); }
int NESTGPU_GetRecSpikeTimes(int i_node, int n, int **n_pt, float ***t_pt) {
  return guard([&] { E().get_rec_spike_times(i_node, n, n_pt, t_pt); return 0; }, 0);
}

// ---- external neurons: not on this path
int NESTGPU_PushSpikesToNodes(int, int *) {
  return guard([&]() -> int { throw NgpuError("ext_neuron is not supported by this engine"); }, 0);
}
int NESTGPU_GetExtNeuronInputSpikes(int *, int **, int **, float **, int) {
  return guard([&]() -> int { throw NgpuError("ext_neuron is not supported by this engine"); }, 0);
}

// ---- group and kernel parameters
int NESTGPU_SetNeuronGroupParam(int i_node, int n, char *name, float val) {
  return guard([&] { E().set_group_param(seq(i_node, n), name, val); return 0; }, 0);
}
int NESTGPU_IsNeuronGroupParam(int i_node, char *name) {
  return guard([&] { return (int)(E().locate(i_node, name) == K_GROUP_PARAM); }, 0);
}
float NESTGPU_GetNeuronGroupParam(int i_node, char *name) {
  return guard([&] { return E().get_group_param(i_node, name); }, 0.0f);
}
int NESTGPU_GetNBoolParam() { return 1; }
char **NESTGPU_GetBoolParamNames() {
  return guard([&] { return name_list({kBoolParam[0]}); }, (char **)nullptr);
}
int NESTGPU_IsBoolParam(char *name) { return idx_of(kBoolParam, 1, name) >= 0; }
int NESTGPU_GetBoolParamIdx(char *name) {
  return guard([&] {
    int i = idx_of(kBoolParam, 1, name);
    if (i < 0) throw NgpuError(std::string("Unrecognized kernel boolean parameter ") + name);
    return i;
  }, 0);
}
bool NESTGPU_GetBoolParam(char *name) {
  return guard([&] {
    if (idx_of(kBoolParam, 1, name) < 0) throw NgpuError(std::string("Unrecognized kernel boolean parameter ") + name);
    return E().print_time;
  }, false);
}
int NESTGPU_SetBoolParam(char *name, bool val) {
  return guard([&] {
    if (idx_of(kBoolParam, 1, name) < 0) throw NgpuError(std::string("Unrecognized kernel boolean parameter ") + name);
    E().print_time = val;
    return 0;
  }, 0);
}
int NESTGPU_GetNFloatParam() { return 3; }
char **NESTGPU_GetFloatParamNames() {
  return guard([&] { return name_list({kFloatParam[0], kFloatParam[1], kFloatParam[2]}); }, (char **)nullptr);
}
int NESTGPU_IsFloatParam(char *name) { return idx_of(kFloatParam, 3, name) >= 0; }
int NESTGPU_GetFloatParamIdx(char *name) {
  return guard([&] {
    int i = idx_of(kFloatParam, 3, name);
    if (i < 0) throw NgpuError(std::string("Unrecognized kernel float parameter ") + name);
    return i;
  }, 0);
}
float NESTGPU_GetFloatParam(char *name) {
  return guard([&] {
    switch (idx_of(kFloatParam, 3, name)) {
    case 0: return E().dt;
    case 1: return E().max_spike_num_fact;
    case 2: return E().max_spike_per_host_fact;
    default: throw NgpuError(std::string("Unrecognized kernel float parameter ") + name);
    }
  }, 0.0f);
}
int NESTGPU_SetFloatParam(char *name, float val) {
  return guard([&] {
    switch (idx_of(kFloatParam, 3, name)) {
    case 0: E().set_time_resolution(val); break;
    case 1: E().max_spike_num_fact = val; break;
    case 2: E().max_spike_per_host_fact = val; break;
    default: throw NgpuError(std::string("Unrecognized kernel float parameter ") + name);
    }
    return 0;
  }, 0);
}
int NESTGPU_GetNIntParam() { return 4; }
char **NESTGPU_GetIntParamNames() {
  return guard([&] { return name_list({kIntParam[0], kIntParam[1], kIntParam[2], kIntParam[3]}); },
               (char **)nullptr);
}
int NESTGPU_IsIntParam(char *name) { return idx_of(kIntParam, 4, name) >= 0; }
int NESTGPU_GetIntParamIdx(char *name) {
  return guard([&] {
    int i = idx_of(kIntParam, 4, name);
    if (i < 0) throw NgpuError(std::string("Unrecognized kernel int parameter ") + name);
    return i;
  }, 0);
}
int NESTGPU_GetIntParam(char *name) {
  return guard([&] {
    switch (idx_of(kIntParam, 4, name)) {
    case 0: return (int)E().seed;
    case 1: return E().verbosity;
    case 2: return E().max_spike_buffer_size;
    case 3: return E().remote_spike_height;
    default: throw NgpuError(std::string("Unrecognized kernel int parameter ") + name);
    }
  }, 0);
}
int NESTGPU_SetIntParam(char *name, int val) {
  return guard([&] {
    switch (idx_of(kIntParam, 4, name)) {
    case 0: E().set_seed((unsigned long long)val); break;
    case 1: E().verbosity = val; break;
    case 2: E().max_spike_buffer_size = val; break;
    case 3: E().remote_spike_height = val; break;
    default: throw NgpuError(std::string("Unrecognized kernel int parameter ") + name);
    }
    return 0;
  }, 0);
}

// ---- engine extensions
void NGPU_FreeArray(void *p) { std::free(p); }

int NGPU_Reset() {
  return guard([&] {
    engine_reset();
    g_conn = ConnSpecC();
    g_syn = SynSpecC();
    return 0;
  }, 0);
}

int NGPU_GetStats(unsigned long long *n_derivs, unsigned long long *n_events, unsigned long long *n_spikes,
                  double *sim_seconds, long long *steps, unsigned int *status) {
  return guard([&] {
    EngineStats s = E().stats();
    g_last_device_ms = s.sim_device_ms;
    if (n_derivs) *n_derivs = s.n_derivs;
    if (n_events) *n_events = s.n_events;
    if (n_spikes) *n_spikes = s.n_spikes;
    if (sim_seconds) *sim_seconds = s.sim_seconds;
    if (steps) *steps = s.steps;
    if (status) *status = s.status;
    return 0;
  }, 0);
}

int NGPU_ConnectArrays(size_t n, int *source, int *target, unsigned char *port, float *weight,
                       float *delay) {
  return guard([&] { E().connect_arrays(n, source, target, port, weight, delay); return 0; }, 0);
}

int NGPU_SetHostRng(int on) {
  return guard([&] {
    E().use_device_rng = (on == 0);
    E().set_seed(E().seed);   // recreate the generator of the chosen kind, same seed
    return 0;
  }, 0);
}

long long NGPU_GetLaunchCount() {
  return guard([&] { return E().n_launches(); }, 0LL);
}

double NGPU_GetSimDeviceMs() {
  return guard([&] { return E().stats().sim_device_ms; }, 0.0);
}

int NGPU_ProfileSteps(int n, double *ms_out) {
  return guard([&] {
    std::vector<double> v = E().profile_steps(n);
    for (size_t i = 0; i < v.size(); i++) ms_out[i] = v[i];
    return (int)v.size();
  }, 0);
}

int NGPU_ConnectFixedIndegreeGPU(int i_source, int n_source, int i_target, int n_target, int indegree,
                                 int port, float weight, float delay_min, float delay_max,
                                 unsigned long long seed) {
  return guard([&] {
    E().connect_fixed_indegree_per_target(i_source, n_source, i_target, n_target, indegree, port, weight,
                                          delay_min, delay_max, seed);
    return 0;
  }, 0);
}

int NGPU_SetPoissonStream(int i_node, int n_node, unsigned int stream) {
  return guard([&] { E().set_poisson_stream(i_node, n_node, stream); return 0; }, 0);
}

int NGPU_GetDeliveryShape(int *n_nodes, int *dmin, int *dspan, long long *n_edges) {
  return guard([&] { E().delivery_shape(n_nodes, dmin, dspan, n_edges); return 0; }, 0);
}

int NGPU_GetDeliveryCsr(long long *seg_off, int *target, unsigned char *port, float *weight) {
  return guard([&] { E().delivery_csr(seg_off, target, port, weight); return 0; }, 0);
}

int NGPU_BuildDeliveryCsr(const int *src, const int *dly, const unsigned *target, const float *weight,
                          size_t n, int n_nodes, int dspan, unsigned long long *seg_off, void *edge,
                          void *stream) {
  return guard([&] {
    if (n_nodes <= 0 || dspan <= 0) throw NgpuError("n_nodes and dspan must be positive");
    if ((n > 0 && (!src || !dly || !target || !weight || !edge)) || !seg_off)
      throw NgpuError("null device pointer");
    pack_delivery_csr(src, dly, target, weight, n, n_nodes, dspan, seg_off, (EdgeW *)edge,
                      (cudaStream_t)stream);
    return 0;
  }, -1);
}

// Same contract as NGPU_BuildDeliveryCsr, scratch from a static device array
// (nest-gpu_b200/csrc/ngpu_noalloc.cu): no device memory is allocated.
int NGPU_BuildDeliveryCsrNoAlloc(const int *src, const int *dly, const unsigned *target, const float *weight,
                                 size_t n, int n_nodes, int dspan, unsigned long long *seg_off, void *edge,
                                 void *stream) {
  return guard([&] {
    if (n_nodes <= 0 || dspan <= 0) throw NgpuError("n_nodes and dspan must be positive");
    if ((n > 0 && (!src || !dly || !target || !weight || !edge)) || !seg_off)
      throw NgpuError("null device pointer");
    pack_delivery_csr_noalloc(src, dly, target, weight, n, n_nodes, dspan, seg_off, (EdgeW *)edge,
                              (cudaStream_t)stream);
    return 0;
  }, -1);
}

int NGPU_SetDeliverBlocks(int n) {
  return guard([&] {
    if (n < 0) throw NgpuError("block count must be >= 0");
    E().deliver_blocks_req = n;
    E().invalidate_graphs();
    return 0;
  }, 0);
}

int NGPU_SetBatchMax(int n) {
  return guard([&] {
    if (n < 1) throw NgpuError("batch length must be >= 1");
    if (E().calibrated()) throw NgpuError("the batch length must be set before calibration");
    E().batch_max = n;
    return 0;
  }, 0);
}

int NGPU_SetRk5Budget(int n) {
  return guard([&] {
    if (n < 0) throw NgpuError("RK5 budget must be >= 0");
    E().rk5_budget = n;
    E().invalidate_graphs();
    return 0;
  }, 0);
}

int NGPU_SetUpdateThreads(int n) {
  return guard([&] {
    if (n != 64 && n != 128 && n != 256) throw NgpuError("update block size must be 64, 128 or 256");
    E().update_threads = n;
    E().invalidate_graphs();
    return 0;
  }, -1);
}

int NGPU_SetDeliverGroup(int g) {
  return guard([&] {
    if (g != 8 && g != 16 && g != 32) throw NgpuError("delivery lane group must be 8, 16 or 32");
    E().deliver_group = g;
    E().invalidate_graphs();
    return 0;
  }, -1);
}

int NGPU_SetUpdateOccupancy(int on) {
  return guard([&] {
    E().update_occupancy = on < 0 ? 0 : (on > 2 ? 2 : on);
    E().invalidate_graphs();
    return 0;
  }, -1);
}

int NGPU_SetDeviceRuleMinEdges(long long n) {
  return guard([&] {
    E().device_rule_min_edges = n;
    return 0;
  }, -1);
}

int NGPU_SetPartition(int rank, int world) {
  return guard([&] { E().set_partition(rank, world); return 0; }, -1);
}

int NGPU_SetExchange(void *send, void *recv, long long cap, int (*exchange)(void *), void *user) {
  return guard([&] { E().set_exchange(send, recv, cap, exchange, user); return 0; }, -1);
}

int NGPU_SetDeliverPrefetch(int on) {
  return guard([&] {
    E().deliver_prefetch = on ? 1 : 0;
    E().invalidate_graphs();
    return 0;
  }, -1);
}

int NGPU_SetDeliverPush(int on) {
  return guard([&] {
    if (E().calibrated())
      throw NgpuError("SetDeliverPush takes effect at calibration: call it before the first Simulate");
    E().deliver_push = on ? 1 : 0;
    return 0;
  }, -1);
}

int NGPU_DeliverPushActive(void) {
  return guard([&] { return E().push_active() ? 1 : 0; }, -1);
}

int NGPU_SetDeliverAggregate(int on) {
  return guard([&] {
    E().deliver_aggregate = on ? 1 : 0;
    E().invalidate_graphs();
    return 0;
  }, -1);
}

int NGPU_SetUpdateTrialIter(int on) {
  return guard([&] {
    E().update_trial_iter = on ? 1 : 0;
    E().invalidate_graphs();
    return 0;
  }, -1);
}

// Test hook: the persistent loop's grid barriers wait for `extra` blocks more than the launch
// has, so their bounded waits run out (the kernel records a timeout and returns).
int NGPU_TestBarrierTimeout(int extra) {
  return guard([&] {
    E().barrier_extra = extra > 0 ? extra : 0;
    return 0;
  }, -1);
}

// Test hook: the training kernel's tensor-core products complete unsignalled, so its bounded
// wait runs out and the call fails.
int NGPU_TestTensorWaitTimeout(int on) {
  return guard([&] {
    set_tensor_wait_test(on);
    return 0;
  }, -1);
}

int NGPU_SetPersistent(int on) {
  return guard([&] {
    E().persistent = on ? 1 : 0;
    E().invalidate_graphs();
    return 0;
  }, -1);
}

int NGPU_SetProgrammaticLaunch(int on) {
  return guard([&] {
    E().launch_pdl = on < 0 ? -1 : (on ? 1 : 0);
    E().invalidate_graphs();
    return 0;
  }, -1);
}

int NGPU_Autotune(int steps, int *update_threads, int *deliver_group, int *deliver_blocks, int *rk5_budget) {
  return guard([&] {
    const int n = E().autotune(steps, nullptr);
    if (update_threads) *update_threads = E().update_threads;
    if (deliver_group) *deliver_group = E().deliver_group;
    if (deliver_blocks) *deliver_blocks = E().deliver_blocks_req;
    if (rk5_budget) *rk5_budget = E().rk5_budget;
    return n;
  }, -1);
}

int NGPU_GetLaunchMapping(int *vals, int n) {
  return guard([&] {
    const int v[10] = {E().update_threads, E().update_occupancy, E().deliver_group, E().deliver_blocks_req,
                       E().rk5_budget, E().persistent, E().launch_pdl, E().update_trial_iter,
                       E().deliver_aggregate, E().deliver_prefetch};
    for (int i = 0; i < n && i < 10; i++) vals[i] = v[i];
    return 10;
  }, -1);
}

double NGPU_MeasureReductionRate(size_t bytes, long long n_ops) {
  return guard([&] { return measure_random_reduction_rate(bytes, n_ops); }, -1.0);
}

int NGPU_GetBatchLength() {
  return guard([&] {
    if (!E().calibrated()) throw NgpuError("the batch length is known after calibration");
    return E().batch_length();
  }, -1);
}

int NGPU_SetGraphSteps(int n) {
  return guard([&] {
    if (n < 1) throw NgpuError("graph steps must be >= 1");
    E().graph_steps = n;
    E().invalidate_graphs();
    return 0;
  }, 0);
}

// ---- learned RK5 step-size proposal
int NGPU_StepModelNParams() { return SM_NPAR; }

int NGPU_Rk5LogStart(long long capacity) {
  return guard([&] { E().rk5_log_start(capacity); return 0; }, -1);
}

int NGPU_Rk5LogStop() {
  return guard([&] { E().rk5_log_stop(); return 0; }, -1);
}

long long NGPU_Rk5LogCount(long long *offered) {
  return guard([&] { return E().rk5_log_count(offered); }, (long long)-1);
}

int NGPU_Rk5LogGet(float *out, long long first, long long n) {
  return guard([&] {
    if (!out && n > 0) throw NgpuError("null output buffer");
    E().rk5_log_get(out, first, n);
    return 0;
  }, -1);
}

int NGPU_StepModelTrain(long long iters, int batch, float lr, float safety, float floor,
                        unsigned long long seed, long long *n_used, float *final_loss) {
  return guard([&] {
    if (iters < 1 || batch < 1 || !(lr > 0.0f) || !(safety > 0.0f) || !(floor >= 0.0f))
      throw NgpuError("invalid training settings");
    TrainConfig c;
    c.iters = iters;
    c.batch = batch;
    c.lr = lr;
    c.safety = safety;
    c.floor = floor;
    c.seed = seed;
    TrainResult r = E().step_model_train(c);
    if (n_used) *n_used = r.n_used;
    if (final_loss) *final_loss = r.final_loss;
    return 0;
  }, -1);
}

int NGPU_StepModelSet(const float *params) {
  return guard([&] {
    if (!params) throw NgpuError("null parameter vector");
    E().step_model_set(params);
    return 0;
  }, -1);
}

int NGPU_StepModelGet(float *params) {
  return guard([&] {
    if (!params) throw NgpuError("null parameter vector");
    E().step_model_get(params);
    return 0;
  }, -1);
}

int NGPU_StepBoundMode(int on) {
  return guard([&] { E().step_bound_mode(on != 0); return 0; }, -1);
}

int NGPU_StepModelEnable(int on) {
  return guard([&] { E().step_model_enable(on != 0); return 0; }, -1);
}

int NGPU_MlpForward(const float *params, const float *feat, int n, float *out) {
  return guard([&] {
    if (n < 0 || !params || (n > 0 && (!feat || !out))) throw NgpuError("invalid arguments");
    mlp_forward_host(params, feat, n, out);
    return 0;
  }, -1);
}

int NGPU_MlpGrad(const float *params, const float *feat, const float *target, int n, float *grad, float *loss) {
  return guard([&] {
    if (n < 1 || !params || !feat || !target || !grad) throw NgpuError("invalid arguments");
    mlp_grad_host(params, feat, target, n, grad, loss);
    return 0;
  }, -1);
}

}  // extern "C"
