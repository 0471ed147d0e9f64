// Host runtime: node groups, parameters, connection store and rules.
// Calibration and the step loop are in ngpu_sim.cpp.
#include "ngpu_engine.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

namespace ngpu {

static const char *kModelName[M_NMODEL] = {
    "aeif_cond_beta_multisynapse", "aeif_cond_alpha_multisynapse", "aeif_psc_exp_multisynapse",
    "aeif_psc_alpha_multisynapse", "iaf_psc_exp", "spike_generator", "poisson_generator",
    "parrot_neuron", "spike_detector"};

static bool is_aeif(int m) { return m <= M_AEIF_PSC_ALPHA; }

// aeif scalar parameter names, reference order (src/aeif_cond_beta_multisynapse_kernel.h:42-58)
enum { A_V_th = 0, A_Delta_T, A_g_L, A_E_L, A_C_m, A_a, A_b, A_tau_w, A_I_e, A_V_peak,
       A_V_reset, A_t_ref, A_refractory_step, A_den_delay, A_NSCAL };
static const char *kAeifScal[A_NSCAL] = {"V_th", "Delta_T", "g_L", "E_L", "C_m", "a", "b",
                                         "tau_w", "I_e", "V_peak", "V_reset", "t_ref",
                                         "refractory_step", "den_delay"};

struct PortShape {
  int npv;
  const char *pv[2];
  int npp;
  const char *pp[4];
};
static PortShape port_shape(int m) {
  switch (m) {
  case M_AEIF_COND_BETA: return {2, {"g", "g1"}, 4, {"E_rev", "tau_rise", "tau_decay", "g0"}};
  case M_AEIF_COND_ALPHA: return {2, {"g", "g1"}, 3, {"E_rev", "tau_syn", "g0", nullptr}};
  case M_AEIF_PSC_EXP: return {1, {"I_syn", nullptr}, 1, {"tau_syn", nullptr, nullptr, nullptr}};
  case M_AEIF_PSC_ALPHA: return {2, {"I_syn", "I1_syn"}, 2, {"tau_syn", "I0", nullptr, nullptr}};
  default: return {0, {nullptr, nullptr}, 0, {nullptr, nullptr, nullptr, nullptr}};
  }
}

enum { I_I_syn_ex = 0, I_I_syn_in, I_V_m_rel, I_refractory_step, I_NVAR };
static const char *kIafVar[I_NVAR] = {"I_syn_ex", "I_syn_in", "V_m_rel", "refractory_step"};
enum { I_tau_m = 0, I_C_m, I_E_L, I_I_e, I_Theta_rel, I_V_reset_rel, I_tau_ex, I_tau_in, I_t_ref,
       I_den_delay, I_P20, I_P11ex, I_P11in, I_P21ex, I_P21in, I_P22, I_NPAR };
static const char *kIafPar[I_NPAR] = {"tau_m", "C_m", "E_L", "I_e", "Theta_rel", "V_reset_rel",
                                      "tau_ex", "tau_in", "t_ref", "den_delay", "P20", "P11ex",
                                      "P11in", "P21ex", "P21in", "P22"};
enum { PG_rate = 0, PG_origin, PG_start, PG_stop, PG_NPAR };
static const char *kPgPar[PG_NPAR] = {"rate", "origin", "start", "stop"};
// parrot_neuron (src/parrot_neuron.cu:40-52)
enum { PR_input_spike_height = 0, PR_dummy_input, PR_V, PR_NVAR };
static const char *kParrotVar[PR_NVAR] = {"input_spike_height", "dummy_input", "V"};
enum { PR_hold_spike_height = 0, PR_den_delay, PR_NPAR };
static const char *kParrotPar[PR_NPAR] = {"hold_spike_height", "den_delay"};
// spike_detector (src/spike_detector.cu:28-70)
enum { SD_input_spike_height = 0, SD_spike_height, SD_NVAR };
static const char *kSdetVar[SD_NVAR] = {"input_spike_height", "spike_height"};
enum { SD_hold_spike_height = 0, SD_NPAR };
static const char *kSdetPar[SD_NPAR] = {"hold_spike_height"};

// one engine per host thread (one network per process as the reference; a test may run
// several partitions of a network side by side in threads of one process)
static thread_local Engine *g_engine = nullptr;

Engine &engine() {
  if (!g_engine) g_engine = new Engine();
  return *g_engine;
}

void engine_reset() {
  delete g_engine;
  g_engine = nullptr;
}

Engine::Engine() {}

Engine::~Engine() {
  if (gen_) curandDestroyGenerator(gen_);
  for (auto &r : records_)
    if (r.fp) fclose(r.fp);
  free_device();
}

void Engine::set_seed(unsigned long long s) {
  // src/nestgpu.cu:182-196: the connection generator gets `s`, device kernels s + 12345
  seed = s;
  kernel_seed = s + 12345ULL;
  if (gen_) {
    curandDestroyGenerator(gen_);
    gen_ = nullptr;
  }
}

void Engine::set_time_resolution(float t) {
  if (calibrated_) throw NgpuError("Time resolution cannot be changed after calibration");
  dt = t;
}

void Engine::make_generator() {
  if (gen_) return;
  int ndev = 0;
  bool dev = use_device_rng && cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0;
  if (!dev) cudaGetLastError();
  curandStatus_t st = dev ? curandCreateGenerator(&gen_, CURAND_RNG_PSEUDO_DEFAULT)
                          : curandCreateGeneratorHost(&gen_, CURAND_RNG_PSEUDO_DEFAULT);
  if (st != CURAND_STATUS_SUCCESS) throw NgpuError("cuRAND generator creation failed");
  gen_device_ = dev;
  curandSetPseudoRandomGeneratorSeed(gen_, seed);
}

// ---------------------------------------------------------------------------
// Random numbers: curandGenerate / GenerateUniform / GenerateNormal on the
// connection generator, one call per request (src/random.cu:8-76).
// ---------------------------------------------------------------------------
template <class T, class F> static std::vector<T> gen_call(bool dev, size_t n, size_t n_alloc, F f) {
  std::vector<T> out(n_alloc);
  if (n_alloc == 0) return out;
  if (dev) {
    T *d = nullptr;
    if (cudaMalloc(&d, n_alloc * sizeof(T)) != cudaSuccess) throw NgpuError("CUDA error");
    curandStatus_t st = f(d);
    cudaDeviceSynchronize();
    cudaMemcpy(out.data(), d, n_alloc * sizeof(T), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (st != CURAND_STATUS_SUCCESS) throw NgpuError("cuRAND error");
  } else {
    if (f(out.data()) != CURAND_STATUS_SUCCESS) throw NgpuError("cuRAND error");
  }
  out.resize(n);
  return out;
}

std::vector<unsigned> Engine::random_int(size_t n) {
  make_generator();
  return gen_call<unsigned>(gen_device_, n, n, [&](unsigned *p) { return curandGenerate(gen_, p, n); });
}

std::vector<float> Engine::random_uniform(size_t n) {
  make_generator();
  return gen_call<float>(gen_device_, n, n, [&](float *p) { return curandGenerateUniform(gen_, p, n); });
}

std::vector<float> Engine::random_normal(size_t n, float mean, float sd) {
  make_generator();
  size_t n1 = (n % 2 == 0) ? n : n + 1;
  return gen_call<float>(gen_device_, n, n1,
                         [&](float *p) { return curandGenerateNormal(gen_, p, n1, mean, sd); });
}

// src/nestgpu.cu:1150-1188: resample out-of-range values from a spare batch,
// optionally snap to a grid of step vstep.
std::vector<float> Engine::random_normal_clipped(size_t n, float mean, float sd, float vmin,
                                                 float vmax, float vstep) {
  const float epsi = 1.0e-6f;
  n = (n / 4 + 1) * 4;
  int n_extra = (int)(n / 10);
  n_extra = (n_extra / 4 + 1) * 4;
  if (n_extra < 1024) n_extra = 1024;
  int i_extra = 0;
  std::vector<float> arr = random_normal(n, mean, sd);
  std::vector<float> extra;
  for (size_t i = 0; i < n; i++) {
    while (arr[i] < vmin || arr[i] > vmax) {
      if (i_extra == 0) extra = random_normal(n_extra, mean, sd);
      arr[i] = extra[i_extra];
      i_extra++;
      if (i_extra == n_extra) i_extra = 0;
    }
  }
  if (vstep > sd * epsi)
    for (size_t i = 0; i < n; i++) arr[i] = vmin + vstep * std::round((arr[i] - vmin) / vstep);
  return arr;
}

// ---------------------------------------------------------------------------
// Nodes
// ---------------------------------------------------------------------------
int Engine::create(const std::string &name, int n, int nport) {
  if (calibrated_) throw NgpuError("Nodes cannot be created after calibration");
  if (n <= 0) throw NgpuError("Number of nodes must be greater than zero.");
  if (nport < 0) throw NgpuError("Number of ports must be >= zero.");
  int m = -1;
  for (int i = 0; i < M_NMODEL; i++)
    if (name == kModelName[i]) m = i;
  if (m < 0) throw NgpuError("Unknown neuron model name: " + name);
  if ((long long)node_group_.size() + n > (1LL << 27)) throw NgpuError("Maximum number of nodes exceeded");
  Group g;
  g.model = m;
  g.i0 = (int)node_group_.size();
  g.n = n;
  if (is_aeif(m)) {
    if (nport > MAX_PORT)
      throw NgpuError("Maximum number of ports " + std::to_string(MAX_PORT) + " exceeded");
    g.nport = nport;
    PortShape s = port_shape(m);
    g.var.assign(2 + s.npv * nport, std::vector<float>(n, 0.0f));
    g.par.assign(A_NSCAL + s.npp * nport, std::vector<float>(n, 0.0f));
    // defaults: src/aeif_cond_beta_multisynapse.cu:37-68 (same for the other aeif models)
    const float d[A_NSCAL] = {-50.4f, 2.0f, 30.0f, -70.6f, 281.0f, 4.0f, 80.5f, 144.0f, 0.0f,
                              0.0f, -60.0f, 0.0f, 0.0f, 0.0f};
    for (int j = 0; j < A_NSCAL; j++) std::fill(g.par[j].begin(), g.par[j].end(), d[j]);
    std::fill(g.var[0].begin(), g.var[0].end(), -70.6f);
    for (int p = 0; p < nport; p++) {
      auto P = [&](int k) -> std::vector<float> & { return g.par[A_NSCAL + s.npp * p + k]; };
      if (m == M_AEIF_COND_BETA) {
        std::fill(P(1).begin(), P(1).end(), 2.0f);
        std::fill(P(2).begin(), P(2).end(), 20.0f);
      } else if (m == M_AEIF_COND_ALPHA) {
        std::fill(P(1).begin(), P(1).end(), 2.0f);
      } else {
        std::fill(P(0).begin(), P(0).end(), 0.2f);
      }
    }
  } else if (m == M_IAF_PSC_EXP) {
    g.nport = 2;
    g.var.assign(I_NVAR, std::vector<float>(n, 0.0f));
    g.par.assign(I_NPAR, std::vector<float>(n, 0.0f));
    // src/iaf_psc_exp.cu:118-175
    const float d[10] = {10.0f, 250.0f, -70.0f, 0.0f, 15.0f, 0.0f, 2.0f, 2.0f, 2.0f, 0.0f};
    for (int j = 0; j < 10; j++) std::fill(g.par[j].begin(), g.par[j].end(), d[j]);
  } else if (m == M_SPIKE_GEN) {
    g.nport = 0;
    g.sg_times.assign(n, {});
    g.sg_heights.assign(n, {});
  } else if (m == M_PARROT) {
    g.nport = 2;
    g.var.assign(PR_NVAR, std::vector<float>(n, 0.0f));
    g.par.assign(PR_NPAR, std::vector<float>(n, 0.0f));
  } else if (m == M_SPIKE_DET) {
    // one input port of weight 1; hold_spike_height defaults to 1 (src/spike_detector.cu:57-70)
    g.nport = 1;
    g.var.assign(SD_NVAR, std::vector<float>(n, 0.0f));
    g.par.assign(SD_NPAR, std::vector<float>(n, 1.0f));
  } else {
    g.nport = 0;
    g.par.assign(PG_NPAR, std::vector<float>(n, 0.0f));
    std::fill(g.par[PG_stop].begin(), g.par[PG_stop].end(), 1.0e30f);
  }
  groups_.push_back(std::move(g));
  node_group_.insert(node_group_.end(), n, (int)groups_.size() - 1);
  order_valid_ = false;
  return groups_.back().i0;
}

int Engine::create_poisson_generator(int n, float rate) {
  int i0 = create("poisson_generator", n, 0);
  std::vector<int> nodes(n);
  std::iota(nodes.begin(), nodes.end(), i0);
  set_scalar(nodes, "rate", rate);
  return i0;
}

int Engine::group_index(int node) {
  if (node < 0 || node >= (int)node_group_.size()) throw NgpuError("Unrecognized node index " + std::to_string(node));
  return node_group_[node];
}

Group &Engine::group_of(int node) { return groups_[group_index(node)]; }

Kind Engine::locate(int node, const std::string &name, int *idx) {
  Group &g = group_of(node);
  int i = -1;
  Kind k = K_NONE;
  if (name == "spike_count" && g.spike_count_on) { k = K_INT_VAR; i = 0; }
  else if (name == "n_rec_spike_times" && g.max_rec > 0) { k = K_INT_VAR; i = 1; }
  else if (is_aeif(g.model)) {
    PortShape s = port_shape(g.model);
    if (name == "V_m") { k = K_SCAL_VAR; i = 0; }
    else if (name == "w") { k = K_SCAL_VAR; i = 1; }
    for (int j = 0; j < s.npv && k == K_NONE; j++) if (name == s.pv[j]) { k = K_PORT_VAR; i = j; }
    for (int j = 0; j < A_NSCAL && k == K_NONE; j++) if (name == kAeifScal[j]) { k = K_SCAL_PARAM; i = j; }
    for (int j = 0; j < s.npp && k == K_NONE; j++) if (name == s.pp[j]) { k = K_PORT_PARAM; i = j; }
    if (k == K_NONE && name == "h_min_rel") { k = K_GROUP_PARAM; i = 0; }
    if (k == K_NONE && name == "h0_rel") { k = K_GROUP_PARAM; i = 1; }
  } else if (g.model == M_IAF_PSC_EXP) {
    for (int j = 0; j < I_NVAR && k == K_NONE; j++) if (name == kIafVar[j]) { k = K_SCAL_VAR; i = j; }
    for (int j = 0; j < I_NPAR && k == K_NONE; j++) if (name == kIafPar[j]) { k = K_SCAL_PARAM; i = j; }
  } else if (g.model == M_POISS_GEN) {
    for (int j = 0; j < PG_NPAR && k == K_NONE; j++) if (name == kPgPar[j]) { k = K_SCAL_PARAM; i = j; }
  } else if (g.model == M_PARROT) {
    for (int j = 0; j < PR_NVAR && k == K_NONE; j++) if (name == kParrotVar[j]) { k = K_SCAL_VAR; i = j; }
    for (int j = 0; j < PR_NPAR && k == K_NONE; j++) if (name == kParrotPar[j]) { k = K_SCAL_PARAM; i = j; }
  } else if (g.model == M_SPIKE_DET) {
    for (int j = 0; j < SD_NVAR && k == K_NONE; j++) if (name == kSdetVar[j]) { k = K_SCAL_VAR; i = j; }
    for (int j = 0; j < SD_NPAR && k == K_NONE; j++) if (name == kSdetPar[j]) { k = K_SCAL_PARAM; i = j; }
  } else if (g.model == M_SPIKE_GEN) {
    if (name == "spike_times") { k = K_ARRAY_PARAM; i = 0; }
    else if (name == "spike_heights") { k = K_ARRAY_PARAM; i = 1; }
  }
  if (idx) *idx = i;
  return k;
}

std::vector<std::string> Engine::names(int node, Kind kind) {
  Group &g = group_of(node);
  std::vector<std::string> r;
  if (kind == K_INT_VAR) {
    if (g.spike_count_on) r.push_back("spike_count");
    if (g.max_rec > 0) r.push_back("n_rec_spike_times");
    return r;
  }
  if (is_aeif(g.model)) {
    PortShape s = port_shape(g.model);
    if (kind == K_SCAL_VAR) r = {"V_m", "w"};
    if (kind == K_PORT_VAR) for (int j = 0; j < s.npv; j++) r.push_back(s.pv[j]);
    if (kind == K_SCAL_PARAM) for (int j = 0; j < A_NSCAL; j++) r.push_back(kAeifScal[j]);
    if (kind == K_PORT_PARAM) for (int j = 0; j < s.npp; j++) r.push_back(s.pp[j]);
    if (kind == K_GROUP_PARAM) r = {"h_min_rel", "h0_rel"};
  } else if (g.model == M_IAF_PSC_EXP) {
    if (kind == K_SCAL_VAR) for (int j = 0; j < I_NVAR; j++) r.push_back(kIafVar[j]);
    if (kind == K_SCAL_PARAM) for (int j = 0; j < I_NPAR; j++) r.push_back(kIafPar[j]);
  } else if (g.model == M_POISS_GEN) {
    if (kind == K_SCAL_PARAM) for (int j = 0; j < PG_NPAR; j++) r.push_back(kPgPar[j]);
  } else if (g.model == M_PARROT) {
    if (kind == K_SCAL_VAR) for (int j = 0; j < PR_NVAR; j++) r.push_back(kParrotVar[j]);
    if (kind == K_SCAL_PARAM) for (int j = 0; j < PR_NPAR; j++) r.push_back(kParrotPar[j]);
  } else if (g.model == M_SPIKE_DET) {
    if (kind == K_SCAL_VAR) for (int j = 0; j < SD_NVAR; j++) r.push_back(kSdetVar[j]);
    if (kind == K_SCAL_PARAM) for (int j = 0; j < SD_NPAR; j++) r.push_back(kSdetPar[j]);
  } else if (g.model == M_SPIKE_GEN) {
    if (kind == K_ARRAY_PARAM) r = {"spike_times", "spike_heights"};
  }
  return r;
}

int Engine::param_size(int node, const std::string &name) {
  int idx;
  Kind k = locate(node, name, &idx);
  Group &g = group_of(node);
  if (k == K_SCAL_PARAM) return 1;
  if (k == K_PORT_PARAM) return g.nport;
  if (k == K_ARRAY_PARAM) {
    int i = node - g.i0;
    return (int)(idx == 0 ? g.sg_times[i].size() : g.sg_heights[i].size());
  }
  throw NgpuError("Unrecognized parameter " + name);
}

int Engine::var_size(int node, const std::string &name) {
  Kind k = locate(node, name);
  if (k == K_SCAL_VAR || k == K_INT_VAR) return 1;
  if (k == K_PORT_VAR) return group_of(node).nport;
  throw NgpuError("Unrecognized variable " + name);
}

// device row of a scalar/port var or of the aeif refractory counter; null if none
static float *dev_row(Group &g, Kind k, int idx, int port) {
  if (!g.d_var) return nullptr;
  if (is_aeif(g.model)) {
    PortShape s = port_shape(g.model);
    if (k == K_SCAL_VAR) return g.d_var + (size_t)idx * g.n;
    if (k == K_PORT_VAR) return g.d_var + (size_t)(2 + s.npv * port + idx) * g.n;
    if (k == K_SCAL_PARAM && idx == A_refractory_step) return g.d_refr;
    return nullptr;
  }
  if ((g.model == M_IAF_PSC_EXP || g.model == M_PARROT || g.model == M_SPIKE_DET) && k == K_SCAL_VAR)
    return g.d_var + (size_t)idx * g.n;
  return nullptr;
}

static std::vector<float> *host_row(Group &g, Kind k, int idx, int port) {
  if (is_aeif(g.model)) {
    PortShape s = port_shape(g.model);
    if (k == K_SCAL_VAR) return &g.var[idx];
    if (k == K_PORT_VAR) return &g.var[2 + s.npv * port + idx];
    if (k == K_SCAL_PARAM) return &g.par[idx];
    if (k == K_PORT_PARAM) return &g.par[A_NSCAL + s.npp * port + idx];
    return nullptr;
  }
  if (k == K_SCAL_VAR) return &g.var[idx];
  if (k == K_SCAL_PARAM) return &g.par[idx];
  return nullptr;
}

// write values (one per listed node) into a row, on the device when it lives there
static void write_row(Group &g, Kind k, int idx, int port, const std::vector<int> &nodes,
                      const std::vector<float> &vals, cudaStream_t st) {
  float *d = dev_row(g, k, idx, port);
  std::vector<float> *h = host_row(g, k, idx, port);
  if (d) {
    // contiguous range: one copy; otherwise read-modify-write of the row
    bool contig = true;
    for (size_t i = 1; i < nodes.size(); i++) contig &= nodes[i] == nodes[0] + (int)i;
    if (contig) {
      cudaMemcpyAsync(d + (nodes[0] - g.i0), vals.data(), vals.size() * sizeof(float),
                      cudaMemcpyHostToDevice, st);
    } else {
      std::vector<float> row(g.n);
      cudaMemcpyAsync(row.data(), d, g.n * sizeof(float), cudaMemcpyDeviceToHost, st);
      cudaStreamSynchronize(st);
      for (size_t i = 0; i < nodes.size(); i++) row[nodes[i] - g.i0] = vals[i];
      cudaMemcpyAsync(d, row.data(), g.n * sizeof(float), cudaMemcpyHostToDevice, st);
    }
    cudaStreamSynchronize(st);
    if (cudaGetLastError() != cudaSuccess) throw NgpuError("CUDA error");
  }
  if (h)
    for (size_t i = 0; i < nodes.size(); i++) (*h)[nodes[i] - g.i0] = vals[i];
  if (k == K_SCAL_PARAM || k == K_PORT_PARAM) g.dirty = true;
}

static void check_same_group(Engine &e, const std::vector<int> &nodes) {
  if (nodes.empty()) throw NgpuError("Empty node list");
  int gi = e.group_index(nodes[0]);
  for (int nd : nodes)
    if (e.group_index(nd) != gi) throw NgpuError("Nodes belong to different node groups in setting parameter");
}

void Engine::set_scalar(const std::vector<int> &nodes, const std::string &name, float v) {
  check_same_group(*this, nodes);
  Group &g = group_of(nodes[0]);
  int idx;
  Kind k = locate(nodes[0], name, &idx);
  if (k == K_GROUP_PARAM) {
    set_group_param(nodes, name, v);
    return;
  }
  if (k != K_SCAL_PARAM && k != K_SCAL_VAR)
    throw NgpuError("Unrecognized scalar parameter or variable " + name);
  if (calibrated_ && k == K_SCAL_PARAM && name == "den_delay")
    throw NgpuError("dendritic delays are fixed at calibration");
  write_row(g, k, idx, 0, nodes, std::vector<float>(nodes.size(), v), stream_);
}

void Engine::set_port_or_array(const std::vector<int> &nodes, const std::string &name, const float *a,
                               int sz) {
  check_same_group(*this, nodes);
  Group &g = group_of(nodes[0]);
  int idx;
  Kind k = locate(nodes[0], name, &idx);
  if (k == K_ARRAY_PARAM) {
    if (calibrated_) throw NgpuError("spike generator times cannot be changed after calibration");
    for (int nd : nodes) {
      int i = nd - g.i0;
      if (idx == 0) g.sg_times[i].assign(a, a + sz);
      else g.sg_heights[i].assign(a, a + sz);
    }
    return;
  }
  if (k != K_PORT_PARAM && k != K_PORT_VAR) throw NgpuError("Unrecognized port parameter or variable " + name);
  if (sz != g.nport)
    throw NgpuError("Parameter array size must be equal to the number of ports of the node group");
  for (int p = 0; p < sz; p++)
    write_row(g, k, idx, p, nodes, std::vector<float>(nodes.size(), a[p]), stream_);
}

void Engine::set_int_var(const std::vector<int> &nodes, const std::string &name, int v) {
  check_same_group(*this, nodes);
  Group &g = group_of(nodes[0]);
  int idx;
  Kind k = locate(nodes[0], name, &idx);
  if (k != K_INT_VAR) throw NgpuError("Unrecognized integer variable " + name);
  int *d = idx == 0 ? g.d_spike_count : g.d_n_rec;
  if (!d) throw NgpuError("integer variable " + name + " is not active on the device yet");
  for (int nd : nodes) cudaMemcpy(d + (nd - g.i0), &v, sizeof(int), cudaMemcpyHostToDevice);
}

std::vector<float> Engine::get_values(const std::vector<int> &nodes, const std::string &name) {
  check_same_group(*this, nodes);
  Group &g = group_of(nodes[0]);
  int idx;
  Kind k = locate(nodes[0], name, &idx);
  if (k == K_GROUP_PARAM) return std::vector<float>(nodes.size(), get_group_param(nodes[0], name));
  if (k == K_INT_VAR) {
    std::vector<int> iv = get_int_values(nodes, name);
    return std::vector<float>(iv.begin(), iv.end());
  }
  int np = (k == K_PORT_PARAM || k == K_PORT_VAR) ? g.nport : 1;
  if (k != K_SCAL_PARAM && k != K_SCAL_VAR && k != K_PORT_PARAM && k != K_PORT_VAR)
    throw NgpuError("Unrecognized parameter or variable " + name);
  std::vector<float> out(nodes.size() * np);
  for (int p = 0; p < np; p++) {
    float *d = dev_row(g, k, idx, p);
    std::vector<float> row;
    if (d) {
      row.resize(g.n);
      cudaStreamSynchronize(stream_);
      if (cudaMemcpy(row.data(), d, g.n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        throw NgpuError("CUDA error");
    } else {
      row = *host_row(g, k, idx, p);
    }
    for (size_t i = 0; i < nodes.size(); i++) out[i * np + p] = row[nodes[i] - g.i0];
  }
  return out;
}

std::vector<int> Engine::get_int_values(const std::vector<int> &nodes, const std::string &name) {
  check_same_group(*this, nodes);
  Group &g = group_of(nodes[0]);
  int idx;
  Kind k = locate(nodes[0], name, &idx);
  if (k != K_INT_VAR) throw NgpuError("Unrecognized integer variable " + name);
  std::vector<int> row(g.n, 0);
  int *d = idx == 0 ? g.d_spike_count : g.d_n_rec;
  if (d) {
    cudaStreamSynchronize(stream_);
    cudaMemcpy(row.data(), d, g.n * sizeof(int), cudaMemcpyDeviceToHost);
  }
  if (idx == 1)   // spike times already drained to the host
    for (int i = 0; i < g.n; i++) row[i] += (int)g.rec_times_host[i].size();
  std::vector<int> out;
  for (int nd : nodes) out.push_back(row[nd - g.i0]);
  return out;
}

void Engine::get_int_values_seq(int i0, int n, const std::string &name, int *out) {
  if (n <= 0) throw NgpuError("Empty node list");
  Group &g = group_of(i0);
  if (group_index(i0 + n - 1) != group_index(i0))
    throw NgpuError("Nodes belong to different node groups in setting parameter");
  int idx;
  Kind k = locate(i0, name, &idx);
  if (k != K_INT_VAR) throw NgpuError("Unrecognized integer variable " + name);
  int *d = idx == 0 ? g.d_spike_count : g.d_n_rec;
  if (d) {
    cudaStreamSynchronize(stream_);
    if (cudaMemcpy(out, d + (i0 - g.i0), (size_t)n * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      throw NgpuError("CUDA error");
  } else {
    std::memset(out, 0, (size_t)n * sizeof(int));
  }
  if (idx == 1)
    for (int i = 0; i < n; i++) out[i] += (int)g.rec_times_host[i0 - g.i0 + i].size();
}

std::vector<float> Engine::get_array_param(int node, const std::string &name) {
  Group &g = group_of(node);
  int idx;
  Kind k = locate(node, name, &idx);
  if (k != K_ARRAY_PARAM) throw NgpuError("Unrecognized array parameter " + name);
  int i = node - g.i0;
  return idx == 0 ? g.sg_times[i] : g.sg_heights[i];
}

void Engine::set_group_param(const std::vector<int> &nodes, const std::string &name, float v) {
  Group &g = group_of(nodes[0]);
  int idx;
  if (locate(nodes[0], name, &idx) != K_GROUP_PARAM) throw NgpuError("Unrecognized neuron group parameter " + name);
  if (nodes.size() != (size_t)g.n || nodes[0] != g.i0)
    throw NgpuError("Group parameters must be set for the whole node group");
  if (idx == 0) g.h_min_rel = v;
  else g.h0_rel = v;
  g.dirty = true;
}

float Engine::get_group_param(int node, const std::string &name) {
  Group &g = group_of(node);
  int idx;
  if (locate(node, name, &idx) != K_GROUP_PARAM) throw NgpuError("Unrecognized neuron group parameter " + name);
  return idx == 0 ? g.h_min_rel : g.h0_rel;
}

// ---------------------------------------------------------------------------
// Synapse groups (src/syn_model.cu:136-238, src/stdp.cu:66-80, src/test_syn_model.cu:42-50)
// ---------------------------------------------------------------------------
static const char *const kStdpParNames[] = {"tau_plus", "tau_minus", "lambda", "alpha", "mu_plus", "mu_minus",
                                            "Wmax"};
static const char *const kTestParNames[] = {"fact", "offset"};

int Engine::create_syn_group(const std::string &model) {
  if (calibrated_) throw NgpuError("Nodes cannot be created after calibration");
  SynGroupDef g;
  if (model == "test_syn_model") {
    g.type = SYN_TEST;
    g.par = {0.1f, 0.0f};
  } else if (model == "stdp") {
    g.type = SYN_STDP;
    g.par = {20.0f, 20.0f, 1.0e-4f, 1.0f, 1.0f, 1.0f, 100.0f};
  } else {
    throw NgpuError("Unknown synapse model name: " + model);
  }
  if (syn_groups_.size() >= 255) throw NgpuError("too many synapse groups");
  syn_groups_.push_back(g);
  return (int)syn_groups_.size();
}

std::vector<std::string> Engine::syn_group_param_names(int g) const {
  if (g < 1 || g > (int)syn_groups_.size()) throw NgpuError("Unrecognized synapse group");
  const SynGroupDef &d = syn_groups_[g - 1];
  const char *const *names = d.type == SYN_STDP ? kStdpParNames : kTestParNames;
  return std::vector<std::string>(names, names + d.par.size());
}

int Engine::syn_group_param_idx(int g, const std::string &name) const {
  const std::vector<std::string> names = syn_group_param_names(g);
  for (size_t i = 0; i < names.size(); i++)
    if (names[i] == name) return (int)i;
  throw NgpuError("Unrecognized parameter " + name);
}

float Engine::get_syn_group_param(int g, const std::string &name) const {
  return syn_groups_[g - 1].par[syn_group_param_idx(g, name)];
}

void Engine::set_syn_group_param(int g, const std::string &name, float v) {
  syn_groups_[g - 1].par[syn_group_param_idx(g, name)] = v;
  if (calibrated_ && plastic_) upload_syn_groups();
}

// ---------------------------------------------------------------------------
// Connections (src/connect.cu:38-74, src/connect_rules.h:161-338)
// ---------------------------------------------------------------------------
void Engine::connect1(int src, int tgt, int port, int syn_group, float w, float d) {
  if (calibrated_) throw NgpuError("Connections cannot be created after calibration");
  if (d < dt) throw NgpuError("Delay must be >= time resolution");
  if (syn_group < 0 || syn_group > (int)syn_groups_.size()) throw NgpuError("Unrecognized synapse group");
  if (port < 0 || port > 255) throw NgpuError("Port index must be >=0");
  if (src < 0 || src >= n_nodes() || tgt < 0 || tgt >= n_nodes()) throw NgpuError("Unrecognized node in connection");
  if (syn_group != 0 || !c_syn_.empty()) {   // the group store exists once a plastic edge does
    c_syn_.resize(c_src_.size(), 0);
    c_syn_.push_back((unsigned char)syn_group);
  }
  c_src_.push_back(src);
  c_tgt_.push_back(tgt);
  c_port_.push_back((unsigned char)port);
  c_w_.push_back(w);
  c_d_.push_back((int)std::round(d / dt) - 1);
  order_valid_ = false;
}

static void cuda_check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw NgpuError(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

template <class T> T *Engine::dcopy(const T *h, size_t n) {
  T *p = nullptr;
  if (cudaMalloc((void **)&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    throw NgpuError("CUDA error: out of device memory for a connection call");
  }
  allocs_.push_back(p);
  if (h && n && cudaMemcpy(p, h, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    throw NgpuError("CUDA error in a connection call");
  return p;
}

// fixed_total_number / fixed_indegree / fixed_outdegree with static synapses and at least
// device_rule_min_edges edges, when the connection generator is cuRAND's device generator:
// the call draws the same random numbers as on the host path (the generator advances the
// same way), keeps them on the device with its weight and delay arrays, and its edges are
// expanded into the delivery layout at calibration (RuleBlockDev, ngpu_build.cu).  Returns
// false (nothing drawn) when the call does not qualify or its arguments need the host path's
// per-edge error reporting.
bool Engine::connect_rule_device(int rule, const int *src_arr, int src0, int ns, const int *tgt_arr, int tgt0,
                                 int nt, int degree, int port, float w, float d, const float *warr,
                                 const float *darr) {
  enum { FIXED_TOTAL_NUMBER = 2, FIXED_INDEGREE = 3, FIXED_OUTDEGREE = 4 };
  if (rule != FIXED_TOTAL_NUMBER && rule != FIXED_INDEGREE && rule != FIXED_OUTDEGREE) return false;
  if (ns <= 0 || nt <= 0 || degree <= 0 || port < 0 || port > 255) return false;
  const size_t n_edges = rule == FIXED_TOTAL_NUMBER ? (size_t)degree
                                                    : (size_t)(rule == FIXED_INDEGREE ? nt : ns) * degree;
  if ((long long)n_edges < device_rule_min_edges) return false;
  const int N = n_nodes();
  for (int i = 0; i < ns; i++) {
    const int s = src_arr ? src_arr[i] : src0 + i;
    if (s < 0 || s >= N || groups_[node_group_[s]].model == M_POISS_GEN) return false;
  }
  for (int i = 0; i < nt; i++) {
    const int t = tgt_arr ? tgt_arr[i] : tgt0 + i;
    if (t < 0 || t >= N) return false;
  }
  // delays: all >= dt (else the host path reports the first offending edge), step range
  int dlo = INT32_MAX, dhi = INT32_MIN;
  if (darr) {
    for (size_t e = 0; e < n_edges; e++) {
      if (!(darr[e] >= dt)) return false;
      const int st = (int)std::round(darr[e] / dt) - 1;
      dlo = std::min(dlo, st);
      dhi = std::max(dhi, st);
    }
  } else {
    if (!(d >= dt)) return false;
    dlo = dhi = (int)std::round(d / dt) - 1;
  }
  make_generator();
  if (!gen_device_) return false;
  const int thresh = 5;
  RuleBlock b;
  b.host_pos = c_src_.size();
  b.dlo = dlo;
  b.dhi = dhi;
  RuleBlockDev &v = b.dev;
  std::memset(&v, 0, sizeof(v));
  v.rule = rule;
  v.ns = ns;
  v.nt = nt;
  v.degree = degree;
  v.port = port;
  v.src0 = src0;
  v.tgt0 = tgt0;
  v.w = w;
  v.d_ms = d;
  v.n_edges = (long long)n_edges;
  v.dt = dt;
  if (rule == FIXED_TOTAL_NUMBER) {
    // the same draw as random_int(2 * degree) on the host path, left on the device
    unsigned *r = dcopy<unsigned>(nullptr, 2 * (size_t)degree);
    if (curandGenerate(gen_, r, 2 * (size_t)degree) != CURAND_STATUS_SUCCESS) throw NgpuError("cuRAND error");
    v.rnd = r;
  } else {
    // one pick shared by all targets (sources), as the host path computes it
    const bool in = rule == FIXED_INDEGREE;
    const int npool = in ? ns : nt;
    if (degree > npool)
      throw NgpuError(in ? "Indegree larger than number of source nodes"
                         : "Outdegree larger than number of target nodes");
    size_t n_rnd = degree;
    if (npool >= thresh * degree) n_rnd *= 5;
    std::vector<unsigned> rnd = random_int(n_rnd);
    std::vector<int> pick;
    if (npool < thresh * degree) {
      pick.resize(npool);
      std::iota(pick.begin(), pick.end(), 0);
      for (int i = 0; i < degree; i++) {
        int j = i + (int)(rnd[i] % (unsigned)(npool - i));
        if (j != i) std::swap(pick[i], pick[j]);
      }
      pick.resize(degree);
    } else {
      std::vector<int> sorted;
      for (int i = 0; i < degree; i++) {
        int i1 = 0, j;
        std::vector<int>::iterator itr;
        do {
          size_t ri = (size_t)i1 * degree + i;
          if (ri >= rnd.size()) throw NgpuError("fixed-degree draw exhausted its random buffer");
          j = (int)(rnd[ri] % (unsigned)npool);
          itr = std::lower_bound(sorted.begin(), sorted.end(), j);
          i1++;
        } while (itr != sorted.end() && *itr == j);
        sorted.insert(itr, j);
        pick.push_back(j);
      }
    }
    v.pick = dcopy<int>(pick.data(), pick.size());
  }
  if (src_arr) {
    b.src_arr.assign(src_arr, src_arr + ns);
    v.src_arr = dcopy<int>(src_arr, ns);
  }
  if (tgt_arr) {
    b.tgt_arr.assign(tgt_arr, tgt_arr + nt);
    v.tgt_arr = dcopy<int>(tgt_arr, nt);
  }
  if (warr) v.warr = dcopy<float>(warr, n_edges);
  if (darr) v.darr = dcopy<float>(darr, n_edges);
  rblocks_.push_back(std::move(b));
  n_rule_edges_ += n_edges;
  order_valid_ = false;
  return true;
}

// Expand the device rule blocks into the host store, each at its place in call order (as
// the host path would have inserted them), for the queries that read the host store.
void Engine::materialize_rule_blocks() {
  if (rblocks_.empty()) return;
  cuda_check(cudaDeviceSynchronize(), "connection store");
  const size_t old_n = c_src_.size();
  std::vector<int> src, tgt, dly;
  std::vector<unsigned char> port, syn;
  std::vector<float> wgt;
  const size_t total = old_n + n_rule_edges_;
  src.reserve(total);
  tgt.reserve(total);
  dly.reserve(total);
  port.reserve(total);
  wgt.reserve(total);
  if (!c_syn_.empty()) syn.reserve(total);
  std::vector<std::pair<size_t, size_t>> shift;   // (old position, edges inserted up to it)
  size_t pos = 0, inserted = 0;
  auto copy_host = [&](size_t upto) {
    for (; pos < upto; pos++) {
      src.push_back(c_src_[pos]);
      tgt.push_back(c_tgt_[pos]);
      dly.push_back(c_d_[pos]);
      port.push_back(c_port_[pos]);
      wgt.push_back(c_w_[pos]);
      if (!c_syn_.empty()) syn.push_back(c_syn_[pos]);
    }
  };
  for (auto &b : rblocks_) {
    copy_host(b.host_pos);
    const RuleBlockDev &v = b.dev;
    const size_t n = (size_t)v.n_edges;
    std::vector<unsigned> rnd;
    std::vector<int> pick;
    std::vector<float> wa, da;
    if (v.rnd) {
      rnd.resize(2 * (size_t)v.degree);
      cuda_check(cudaMemcpy(rnd.data(), v.rnd, rnd.size() * sizeof(unsigned), cudaMemcpyDeviceToHost), "rnd");
    } else {
      pick.resize(v.degree);
      cuda_check(cudaMemcpy(pick.data(), v.pick, pick.size() * sizeof(int), cudaMemcpyDeviceToHost), "pick");
    }
    if (v.warr) {
      wa.resize(n);
      cuda_check(cudaMemcpy(wa.data(), v.warr, n * sizeof(float), cudaMemcpyDeviceToHost), "weights");
    }
    if (v.darr) {
      da.resize(n);
      cuda_check(cudaMemcpy(da.data(), v.darr, n * sizeof(float), cudaMemcpyDeviceToHost), "delays");
    }
    auto S = [&](int i) { return b.src_arr.empty() ? v.src0 + i : b.src_arr[i]; };
    auto T = [&](int i) { return b.tgt_arr.empty() ? v.tgt0 + i : b.tgt_arr[i]; };
    for (size_t e = 0; e < n; e++) {
      int is, it;
      if (v.rule == 2) {
        is = (int)(rnd[2 * e] % (unsigned)v.ns);
        it = (int)(rnd[2 * e + 1] % (unsigned)v.nt);
      } else {
        const size_t kk = e / v.degree;
        const int i = (int)(e - kk * v.degree);
        if (v.rule == 3) { is = pick[i]; it = (int)kk; } else { is = (int)kk; it = pick[i]; }
      }
      src.push_back(S(is));
      tgt.push_back(T(it));
      port.push_back((unsigned char)v.port);
      wgt.push_back(v.warr ? wa[e] : v.w);
      dly.push_back((int)std::round((v.darr ? da[e] : v.d_ms) / dt) - 1);
      if (!c_syn_.empty()) syn.push_back(0);
    }
    inserted += n;
    shift.push_back({b.host_pos, inserted});
  }
  copy_host(old_n);
  // host-edge ids held elsewhere (plastic entries) move by the edges inserted before them
  for (auto &pe : pl_of_edge_) {
    size_t add = 0;
    for (auto &sh : shift)
      if (sh.first <= pe.first) add = sh.second;
    pe.first += add;
  }
  c_src_.swap(src);
  c_tgt_.swap(tgt);
  c_d_.swap(dly);
  c_port_.swap(port);
  c_w_.swap(wgt);
  if (!c_syn_.empty()) c_syn_.swap(syn);
  rblocks_.clear();
  n_rule_edges_ = 0;
  order_valid_ = false;
}

void Engine::connect_rule(int rule, const int *src_arr, int src0, int ns, const int *tgt_arr, int tgt0,
                          int nt, int degree, int port, int syn_group, float w, float d,
                          const float *warr, const float *darr) {
  if (calibrated_) throw NgpuError("Connections cannot be created after calibration");
  if (syn_group == 0 && connect_rule_device(rule, src_arr, src0, ns, tgt_arr, tgt0, nt, degree, port, w, d,
                                            warr, darr))
    return;
  auto S = [&](int i) { return src_arr ? src_arr[i] : src0 + i; };
  auto T = [&](int i) { return tgt_arr ? tgt_arr[i] : tgt0 + i; };
  auto one = [&](int is, int itn, size_t ia) {
    connect1(S(is), T(itn), port, syn_group, warr ? warr[ia] : w, darr ? darr[ia] : d);
  };
  enum { ONE_TO_ONE = 0, ALL_TO_ALL, FIXED_TOTAL_NUMBER, FIXED_INDEGREE, FIXED_OUTDEGREE };
  const int thresh = 5;
  switch (rule) {
  case ONE_TO_ONE:
    if (ns != nt) throw NgpuError("Number of source and target nodes must be equal for the one-to-one connection rule");
    for (int i = 0; i < ns; i++) one(i, i, (size_t)i);
    break;
  case ALL_TO_ALL:
    for (int itn = 0; itn < nt; itn++)
      for (int isn = 0; isn < ns; isn++) one(isn, itn, (size_t)itn * ns + isn);
    break;
  case FIXED_TOTAL_NUMBER: {
    std::vector<unsigned> rnd = random_int(2 * (size_t)degree);
    for (int i = 0; i < degree; i++) one((int)(rnd[2 * i] % ns), (int)(rnd[2 * i + 1] % nt), (size_t)i);
    break;
  }
  case FIXED_INDEGREE:
  case FIXED_OUTDEGREE: {
    // One random draw per call; every target (source) gets the same pick, as the
    // reference does (THREAD_MAXNUM == 1, src/connect_rules.h:214-262).
    const bool in = rule == FIXED_INDEGREE;
    const int npool = in ? ns : nt, nloop = in ? nt : ns;
    if (degree > npool)
      throw NgpuError(in ? "Indegree larger than number of source nodes"
                         : "Outdegree larger than number of target nodes");
    size_t n_rnd = degree;
    if (npool >= thresh * degree) n_rnd *= 5;
    std::vector<unsigned> rnd = random_int(n_rnd);
    for (int kk = 0; kk < nloop; kk++) {
      std::vector<int> pick;
      if (npool < thresh * degree) {
        pick.resize(npool);
        std::iota(pick.begin(), pick.end(), 0);
        for (int i = 0; i < degree; i++) {
          int j = i + (int)(rnd[i] % (unsigned)(npool - i));
          if (j != i) std::swap(pick[i], pick[j]);
        }
      } else {
        std::vector<int> sorted;
        for (int i = 0; i < degree; i++) {
          int i1 = 0, j;
          std::vector<int>::iterator itr;
          do {
            size_t ri = (size_t)i1 * degree + i;
            if (ri >= rnd.size()) throw NgpuError("fixed-degree draw exhausted its random buffer");
            j = (int)(rnd[ri] % (unsigned)npool);
            itr = std::lower_bound(sorted.begin(), sorted.end(), j);
            i1++;
          } while (itr != sorted.end() && *itr == j);
          sorted.insert(itr, j);
          pick.push_back(j);
        }
      }
      for (int i = 0; i < degree; i++) {
        if (in) one(pick[i], kk, (size_t)kk * degree + i);
        else one(kk, pick[i], (size_t)kk * degree + i);
      }
    }
    break;
  }
  default: throw NgpuError("Unknown connection rule");
  }
}

// Fixed in-degree with per-target random sources (with replacement) and delays uniform on
// the time grid in [dmin_ms, dmax_ms], generated on the device at calibration.  Unlike the
// reference's fixed_indegree rule every target draws its own sources.
void Engine::connect_fixed_indegree_per_target(int src0, int ns, int tgt0, int nt, int k, int port,
                                               float w, float dmin_ms, float dmax_ms, uint64_t s) {
  if (calibrated_) throw NgpuError("Connections cannot be created after calibration");
  if (ns <= 0 || nt <= 0 || k <= 0) throw NgpuError("empty connection block");
  if (src0 < 0 || src0 + ns > n_nodes()) throw NgpuError("Unrecognized source node");
  Group &tg = group_of(tgt0);
  if (tgt0 + nt > tg.i0 + tg.n) throw NgpuError("Targets of a generated block must belong to one node group");
  if (port < 0 || port >= tg.nport) throw NgpuError("Port index out of range");
  if (dmin_ms < dt || dmax_ms < dmin_ms) throw NgpuError("Delay must be >= time resolution");
  for (int i = src0; i < src0 + ns; i++)
    if (groups_[node_group_[i]].model == M_POISS_GEN) throw NgpuError("poisson_generator cannot be a source of a generated block");
  if ((long long)nt * k > (1LL << 40)) throw NgpuError("connection block too large");
  blocks_.push_back({src0, ns, tgt0, nt, k, port, w, dmin_ms, dmax_ms, s});
  n_generated_ += (size_t)nt * k;
}

void Engine::set_poisson_stream(int i0, int n, uint32_t stream0) {
  if (calibrated_) throw NgpuError("Poisson streams must be set before calibration");
  if (n <= 0) return;
  Group &g = group_of(i0);
  if (g.model != M_POISS_GEN) throw NgpuError("Poisson streams apply to poisson_generator nodes only");
  if (i0 + n > g.i0 + g.n) throw NgpuError("Poisson stream range crosses a node group");
  if (g.pg_stream.empty()) {
    // untouched generators keep their default: the index among all generators, known at
    // calibration; mark them with the default computed there
    g.pg_stream.assign(g.n, 0xffffffffu);
  }
  for (int j = 0; j < n; j++) g.pg_stream[i0 - g.i0 + j] = stream0 + (uint32_t)j;
}

void Engine::connect_arrays(size_t n, const int *src, const int *tgt, const unsigned char *port,
                            const float *w, const float *d) {
  if (calibrated_) throw NgpuError("Connections cannot be created after calibration");
  size_t base = c_src_.size();
  c_src_.resize(base + n);
  c_tgt_.resize(base + n);
  c_port_.resize(base + n);
  c_w_.resize(base + n);
  c_d_.resize(base + n);
  if (!c_syn_.empty()) c_syn_.resize(base + n, 0);
  const int N = n_nodes();
  for (size_t i = 0; i < n; i++) {
    if (src[i] < 0 || src[i] >= N || tgt[i] < 0 || tgt[i] >= N) throw NgpuError("Unrecognized node in connection");
    if (d[i] < dt) throw NgpuError("Delay must be >= time resolution");
    c_src_[base + i] = src[i];
    c_tgt_[base + i] = tgt[i];
    c_port_[base + i] = port ? port[i] : 0;
    c_w_[base + i] = w[i];
    c_d_[base + i] = (int)std::round(d[i] / dt) - 1;
  }
  order_valid_ = false;
}

// Reference order: sources ascending, delay groups ascending, insertion order.
void Engine::build_order() {
  materialize_rule_blocks();
  if (order_valid_) return;
  const size_t E = c_src_.size();
  const int N = n_nodes();
  std::vector<long long> cnt(N + 1, 0);
  for (size_t e = 0; e < E; e++) cnt[c_src_[e] + 1]++;
  for (int i = 0; i < N; i++) cnt[i + 1] += cnt[i];
  src_first_ = cnt;
  ord_.assign(E, 0);
  std::vector<long long> pos(cnt.begin(), cnt.end() - 1);
  for (size_t e = 0; e < E; e++) ord_[pos[c_src_[e]]++] = (long long)e;
  ord_grp_.assign(E, 0);
  ord_idx_.assign(E, 0);
  for (int s = 0; s < N; s++) {
    long long a = cnt[s], b = cnt[s + 1];
    if (b - a > 1)
      std::stable_sort(ord_.begin() + a, ord_.begin() + b,
                       [&](long long x, long long y) { return c_d_[x] < c_d_[y]; });
    int grp = -1, idx = 0, last = INT32_MIN;
    for (long long p = a; p < b; p++) {
      int dd = c_d_[ord_[p]];
      if (dd != last) { grp++; idx = 0; last = dd; }
      ord_grp_[p] = grp;
      ord_idx_[p] = idx++;
    }
  }
  order_valid_ = true;
}

std::vector<int> Engine::get_connections(const int *src_arr, int src0, int ns, const int *tgt_arr,
                                         int tgt0, int nt, int syn_group) {
  build_order();
  std::vector<int> tsorted;
  if (tgt_arr) {
    tsorted.assign(tgt_arr, tgt_arr + nt);
    std::sort(tsorted.begin(), tsorted.end());
  }
  const int N = n_nodes();
  std::vector<int> out;
  auto want_t = [&](int t) {
    if (nt < 0) return true;   // no target filter
    if (tgt_arr) return std::binary_search(tsorted.begin(), tsorted.end(), t);
    return t >= tgt0 && t < tgt0 + nt;
  };
  int ns_eff = ns < 0 ? N : ns;
  for (int is = 0; is < ns_eff; is++) {
    int s = ns < 0 ? is : (src_arr ? src_arr[is] : src0 + is);
    if (s < 0 || s >= N) throw NgpuError("Unrecognized source node");
    for (long long p = src_first_[s]; p < src_first_[s + 1]; p++) {
      if (want_t(c_tgt_[ord_[p]]) && (syn_group < 0 || syn_of(ord_[p]) == syn_group)) {
        out.push_back(s);
        out.push_back(ord_grp_[p]);
        out.push_back(ord_idx_[p]);
      }
    }
  }
  return out;
}

void Engine::connection_status(int src, int grp, int idx, int *tgt, unsigned char *port,
                               unsigned char *syn, float *delay, float *w) {
  build_order();
  if (src < 0 || src >= n_nodes()) throw NgpuError("Unrecognized source node");
  for (long long p = src_first_[src]; p < src_first_[src + 1]; p++) {
    if (ord_grp_[p] == grp && ord_idx_[p] == idx) {
      long long e = ord_[p];
      *tgt = c_tgt_[e];
      *port = c_port_[e];
      *syn = syn_of(e);
      *delay = dt * (float)(c_d_[e] + 1);
      *w = c_w_[e];
      if (*syn && calibrated_) *w = plastic_weight((size_t)e, *w);   // it lives on the device
      return;
    }
  }
  throw NgpuError("Connection not found");
}

// ---------------------------------------------------------------------------
// Recording options
// ---------------------------------------------------------------------------
int Engine::create_record(const std::string &file, const std::vector<std::string> &vars,
                          const std::vector<int> &nodes, const std::vector<int> &ports) {
  if (calibrated_) throw NgpuError("Records must be created before calibration");
  RecordSpec r;
  r.file = file;
  r.var = vars;
  r.node = nodes;
  r.port = ports;
  for (size_t i = 0; i < nodes.size(); i++) {
    if (vars[i] == "spike") { group_of(nodes[i]); continue; }
    Kind k = locate(nodes[i], vars[i]);
    if (k != K_SCAL_VAR && k != K_PORT_VAR && !(k == K_SCAL_PARAM && vars[i] == "refractory_step"))
      throw NgpuError("Unrecognized variable " + vars[i]);
    if (k == K_PORT_VAR && (ports[i] < 0 || ports[i] >= group_of(nodes[i]).nport))
      throw NgpuError("Port index out of range in record");
  }
  records_.push_back(std::move(r));
  return (int)records_.size() - 1;
}

RecordSpec &Engine::record(int i) {
  if (i < 0 || i >= (int)records_.size()) throw NgpuError("Record does not exist.");
  return records_[i];
}

void Engine::activate_spike_count(int i_node, int n) {
  Group &g = group_of(i_node);
  (void)n;
  if (g.spike_count_on) throw NgpuError("Spike count already activated");
  if (calibrated_) throw NgpuError("Spike count must be activated before calibration");
  g.spike_count_on = true;
}

void Engine::activate_rec_spike_times(int i_node, int n, int max_n) {
  Group &g = group_of(i_node);
  (void)n;
  if (max_n <= 0) throw NgpuError("Maximum number of recorded spike times must be greater than 0");
  if (g.max_rec > 0) throw NgpuError("Spike times recording already activated");
  if (calibrated_) throw NgpuError("Spike times recording must be activated before calibration");
  g.max_rec = max_n;
  g.rec_times_host.assign(g.n, {});
}

void Engine::set_rec_spike_times_step(int i_node, int n, int step) {
  Group &g = group_of(i_node);
  (void)n;
  g.rec_times_step = step;
}

int Engine::n_rec_spike_times(int node) {
  Group &g = group_of(node);
  if (g.max_rec <= 0) throw NgpuError("Spike times recording was not activated");
  return get_int_values({node}, "n_rec_spike_times")[0];
}

void Engine::get_rec_spike_times(int i_node, int n, int **n_pt, float ***t_pt) {
  Group &g = group_of(i_node);
  if (g.max_rec <= 0) throw NgpuError("Spike times recording was not activated");
  drain_rec_spike_times();
  int r0 = i_node - g.i0;
  if (r0 < 0 || r0 + n > g.n) throw NgpuError("Nodes belong to different node groups");
  // like BaseNeuron::GetRecSpikeTimes (src/base_neuron.cu:1528-1580): each call hands out
  // the spike times buffered since the previous call
  g.rec_export.assign(n, {});
  g.rec_n_host.assign(n, 0);
  g.rec_ptr_host.assign(n, nullptr);
  for (int i = 0; i < n; i++) {
    g.rec_export[i].swap(g.rec_times_host[r0 + i]);
    g.rec_n_host[i] = (int)g.rec_export[i].size();
    g.rec_ptr_host[i] = g.rec_export[i].data();
  }
  *n_pt = g.rec_n_host.data();
  *t_pt = g.rec_ptr_host.data();
}

}  // namespace ngpu
