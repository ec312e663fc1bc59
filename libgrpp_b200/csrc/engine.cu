// GRPP engine: the single CUDA translation unit (device tables, kernels, host
// orchestration of a batch of (shell A, shell B, centre C) tasks).
//
// Pipeline of one batch (kernels and uploads on the state's stream; the batched call's
// downloads of finished chunks on a second stream):
//   1. atab_kernel    k-independent angular tensors, cached per device and (L, l)
//   2. mmd_kernel     type 1 blocks <A|U_L|B> written straight into the arep output,
//                     and <S|U_oc|oc>, <S|oc> Cartesian blocks for every (shell, centre)
//                     that needs outercore projections
//   3. oc_proj_kernel Cartesian -> real spherical transform of those blocks
//   4. radial kernels Q tables of every semilocal potential of every task: screening,
//                     then (learned mode) the level model orders the tasks deepest
//                     predicted level first, then the grid walk
//   5. final_kernel   per task: T1 + sum type 2 + sum 2/(2L+1) SO + outercore, in
//                     libgrpp_full_grpp_integrals' accumulation order
// mmd_kernel and final_kernel run persistent grids that pop work from a queue ordered by
// estimated work, largest first; the walk does the same in learned mode.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "grpp_common.cuh"
#include "specfunc.cuh"
#define GRPP_NO_RADIAL_TABLE_KERNELS  // ftab_kernel, wu_table_kernel: compiled in nofma.cu
#include "radial.cuh"
#include "mmd.cuh"
#define GRPP_NO_ANGULAR_KERNELS  // the angular kernels are compiled in nofma.cu (no contraction)
#include "angular.cuh"
#include "nofma_launch.h"
#include "level_model.cuh"
#include "gradient.cuh"
#include "onee.cuh"
#include "tables.h"
#include "engine.h"

namespace grpp {

constexpr size_t kFinSmemMax = 220 * 1024;  // dynamic shared memory of the assembly kernel (+ its static 3 kB)

// ------------------------------------------------------------------ errors
namespace {
thread_local int t_err = 0;
thread_local std::string t_msg;
}  // namespace

void set_error(int code, const std::string &msg)
{
    t_err = code;
    t_msg = msg;
}
int last_error() { return t_err; }
const char *last_error_message() { return t_msg.c_str(); }

#define GRPP_CUDA(call)                                                                           \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            set_error(LIBGRPP_B200_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
            return LIBGRPP_B200_ERR_CUDA;                                                         \
        }                                                                                         \
    } while (0)

// ------------------------------------------------------------------ device state
namespace {

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n)
    {
        if (n <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(n, 1 << 20);
        want = want + want / 4;
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
};

// page-locked host staging buffer (uploads that do not wait for the stream)
struct PinBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n)
    {
        if (n <= cap) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        const size_t want = std::max<size_t>(n + n / 4, 1 << 20);
        cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
        if (e == cudaSuccess) cap = want;
        return e;
    }
};

// Two buffer sets: a batch larger than one chunk alternates between them, so the host
// prepares and uploads chunk c+1 and downloads chunk c-1 while the GPU runs chunk c.
struct DeviceState {
    int device = -1;
    int nsm = 148;                       // multiprocessors of the device (set at initialisation)
    bool ready = false;
    cudaStream_t stream = nullptr;       // all kernels and uploads
    cudaStream_t copy_stream = nullptr;  // downloads of finished chunks
    cudaEvent_t ev[2][6];                // per buffer set: phase boundaries of one execution
    cudaEvent_t done[2];                 // per buffer set: execution and its status copy finished
    cudaEvent_t uploaded[2];             // per buffer set: the staging buffer's last upload finished
    std::vector<void *> table_bufs;
    DevBuf in[2], scratch[2], out[2];
    PinBuf stage[2];                     // upload staging per buffer set
    int *hstat[2] = {nullptr, nullptr};  // page-locked status words + counters per buffer set
    DevBuf atab;
    size_t atab_used = 0;
    DevBuf grad;  // density-contracted gradient: tasks, component table, D, per-task sums
    DevBuf onee;  // one-electron batches: inputs, angular factors, outputs
    const double *fermi = nullptr;  // S_j table of the Fermi nuclear models
    // learned grid-level model (libgrpp_b200_set_level_model): FP32 normalisation, BF16 weights
    float *lm_norm = nullptr;
    __nv_bfloat16 *lm_w = nullptr;
    bool lm_ready = false;
    std::vector<int64_t> atab_off;
    bool atab_dirty = true;  // atab_off has entries the device copy lacks
    DevBuf atab_off_dev;
    std::vector<cudaEvent_t> gev[2];     // per buffer set: boundaries of the assembly launches (autotuning)
    std::map<int, int> fin_tune;         // assembly class -> block size picked by the autotuner
    std::mutex mu;
};

std::mutex g_state_mu;
DeviceState g_states[64];
HostTables g_host;
bool g_host_ready = false;

template <typename T>
cudaError_t upload_vec(DeviceState &st, const std::vector<T> &v, const T **out)
{
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(v.size(), 1) * sizeof(T));
    if (e != cudaSuccess) return e;
    st.table_bufs.push_back(p);
    if (!v.empty()) e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    *out = (const T *)p;
    return e;
}

int init_device_state(DeviceState &st, int device)
{
    if (!g_host_ready) {
        build_host_tables(g_host);
        g_host_ready = true;
    }
    const HostTables &h = g_host;
    DeviceTables d;
    GRPP_CUDA(upload_vec(st, h.bessel, &d.bessel));
    GRPP_CUDA(upload_vec(st, h.bessel_p, &d.bessel_p));
    GRPP_CUDA(upload_vec(st, h.rfun, &d.rfun));
    GRPP_CUDA(upload_vec(st, h.boys, &d.boys));
    GRPP_CUDA(upload_vec(st, h.dawson, &d.dawson));
    GRPP_CUDA(upload_vec(st, h.rsh_coef, &d.rsh_coef));
    GRPP_CUDA(upload_vec(st, h.rsh_off, &d.rsh_off));
    GRPP_CUDA(upload_vec(st, h.rsh_comb, &d.rsh_comb));
    GRPP_CUDA(upload_vec(st, h.rsh_comb_off, &d.rsh_comb_off));
    GRPP_CUDA(upload_vec(st, h.lmat, &d.lmat));
    GRPP_CUDA(upload_vec(st, h.lmat_off, &d.lmat_off));
    GRPP_CUDA(upload_vec(st, h.dfact, &d.dfact));
    GRPP_CUDA(upload_vec(st, h.binom, &d.binom));
    GRPP_CUDA(upload_vec(st, h.grid, &d.grid));
    GRPP_CUDA(upload_vec(st, h.fermi, &st.fermi));
    GRPP_CUDA(cudaMemcpyToSymbol(c_tab, &d, sizeof(d)));
    GRPP_CUDA(ang_upload_tables(&d, sizeof(d)));
    GRPP_CUDA(cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking));
    GRPP_CUDA(cudaStreamCreateWithFlags(&st.copy_stream, cudaStreamNonBlocking));
    for (int k = 0; k < 2; k++) {
        for (auto &e : st.ev[k]) GRPP_CUDA(cudaEventCreate(&e));
        GRPP_CUDA(cudaEventCreateWithFlags(&st.done[k], cudaEventDisableTiming));
        GRPP_CUDA(cudaEventCreateWithFlags(&st.uploaded[k], cudaEventDisableTiming));
        GRPP_CUDA(cudaHostAlloc((void **)&st.hstat[k], 16 * sizeof(int) + kRadCntNum * sizeof(unsigned long long),
                                cudaHostAllocDefault));
    }
    st.atab_off.assign((kMaxL + 2) * (kMaxL + 2), -1);
    GRPP_CUDA(cudaFuncSetAttribute(mmd_kernel<8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    GRPP_CUDA(cudaFuncSetAttribute(mmd_kernel<32, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    GRPP_CUDA(cudaFuncSetAttribute(mmd_kernel<8, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    GRPP_CUDA(cudaFuncSetAttribute(mmd_kernel<32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    GRPP_CUDA(cudaFuncSetAttribute(radial_walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    GRPP_CUDA(ang_set_final_max_smem((int)kFinSmemMax));
    GRPP_CUDA(cudaFuncSetAttribute(type1_num_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(t1_smem_doubles(kT1MaxLam) * sizeof(double))));
    GRPP_CUDA(cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp_train_smem_bytes()));
    GRPP_CUDA(cudaDeviceGetAttribute(&st.nsm, cudaDevAttrMultiProcessorCount, device));
    st.device = device;
    st.ready = true;
    return 0;
}

DeviceState *get_state(int &rc)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(LIBGRPP_B200_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        rc = LIBGRPP_B200_ERR_CUDA;
        return nullptr;
    }
    if (dev < 0 || dev >= 64) {
        set_error(LIBGRPP_B200_ERR_CUDA, "device index out of range");
        rc = LIBGRPP_B200_ERR_CUDA;
        return nullptr;
    }
    DeviceState &st = g_states[dev];
    std::lock_guard<std::mutex> lk(g_state_mu);
    if (!st.ready) {
        rc = init_device_state(st, dev);
        if (rc) return nullptr;
    }
    rc = 0;
    return &st;
}

// ------------------------------------------------------------------ host packing
struct Packer {
    std::vector<char> buf;
    template <typename T>
    size_t add(const std::vector<T> &v)
    {
        size_t off = (buf.size() + 255) & ~size_t(255);
        buf.resize(off + std::max<size_t>(v.size(), 1) * sizeof(T));
        if (!v.empty()) memcpy(buf.data() + off, v.data(), v.size() * sizeof(T));
        return off;
    }
};

// Slot schedule of the Cartesian pairs of one (bra, ket) table class for mmd_kernel. Pairs
// with equal (tx, uy, vz) = (ax+bx, ay+by, az+bz) have the same contraction loops: they are
// coupled two by two into slots (2h, 2h+1) of one lane (an odd one out takes a slot couple
// alone), and the couples fill the slot rows in (tx, uy, vz) order, so the 32 lanes of a row
// run equal or nearly equal loops. Appends 32 x kpl slots to out; returns the rows in use.
static int mmd_pair_schedule(const int8_t *ca, int nA, const int8_t *cb, int nB, int kpl, std::vector<uint16_t> &out)
{
    std::map<int, std::vector<int>> groups;  // key (tx * 32 + uy) * 32 + vz, ascending
    for (int m = 0; m < nA; m++)
        for (int n = 0; n < nB; n++) {
            const int tx = ca[3 * m] + cb[3 * n], uy = ca[3 * m + 1] + cb[3 * n + 1], vz = ca[3 * m + 2] + cb[3 * n + 2];
            groups[(tx * 32 + uy) * 32 + vz].push_back(m * nB + n);
        }
    std::vector<std::pair<int, int>> units;
    for (auto &g : groups)
        for (size_t i = 0; i < g.second.size(); i += 2)
            units.push_back({g.second[i], i + 1 < g.second.size() ? g.second[i + 1] : -1});
    const size_t base = out.size();
    out.resize(base + 32 * (size_t)kpl, kMmdNoPair);
    if ((int)units.size() > 16 * kpl) {  // more units than slot couples: plain order, unequal couples
        for (int pr = 0; pr < nA * nB; pr++) out[base + pr] = (uint16_t)pr;
        return (nA * nB + 63) / 64;
    }
    for (size_t r = 0; r < units.size(); r++) {
        const int row = (int)(r / 32), lane = (int)(r % 32);
        out[base + (2 * row) * 32 + lane] = (uint16_t)units[r].first;
        if (units[r].second >= 0) out[base + (2 * row + 1) * 32 + lane] = (uint16_t)units[r].second;
    }
    return (int)(units.size() + 31) / 32;
}

// Update programs of mmd_kernel's Hermite coefficients for every (la, lb) with la, lb <= lmax,
// and of its R^n_tuv tables for every S = 1..smax (mmd_e_code / MmdArgs::rtab).
static void mmd_update_tables(int lmax, int smax, std::vector<int> &etab, std::vector<int> &etab_off,
                              std::vector<int2> &rtab, std::vector<int> &rtab_off)
{
    etab_off.assign((kMaxL + 1) * (kMaxL + 1), 0);
    for (int la = 0; la <= lmax; la++)
        for (int lb = 0; lb <= lmax; lb++) {
            etab_off[la * (kMaxL + 1) + lb] = (int)etab.size();
            const int S = la + lb, la1 = la + 1, lb1 = lb + 1, S1 = S + 1;
            for (int w = 0; w <= S; w++) {
                const int ilo = std::max(0, w - lb), ihi = std::min(la, w), per_axis = (ihi - ilo + 1) * (w + 1);
                for (int e = 0; e < 3 * per_axis; e++) {
                    const int ax = e / per_axis, r = e % per_axis, i = ilo + r / (w + 1), t = r % (w + 1), j = w - i;
                    etab.push_back(mmd_e_code(((ax * la1 + i) * lb1 + j) * S1 + t, ax, i, j, t));
                }
            }
        }
    rtab_off.assign(2 * kMaxL + 1, 0);
    for (int S = 1; S <= smax; S++) {
        rtab_off[S] = (int)rtab.size();
        std::vector<int> lvl(S + 1);
        for (int s = 0, o = 0; s <= S; s++) {
            lvl[s] = o;
            o += (s + 1) * (s + 2) / 2 * (S - s + 1);
        }
        rtab.resize(rtab.size() + mmd_r_size(S), int2{0, 0});
        int2 *tab = rtab.data() + rtab_off[S];
        for (int s = 1; s <= S; s++) {
            const int ne = (s + 1) * (s + 2) / 2, nn = S - s + 1, ne1 = s * (s + 1) / 2, ne2 = (s - 1) * s / 2;
            const int o1 = lvl[s - 1], o2 = s >= 2 ? lvl[s - 2] : 0;
            for (int e = 0; e < ne * nn; e++) {
                const int n = e / ne, idx = e % ne;
                int kk = 0;
                while ((kk + 1) * (kk + 2) / 2 <= idx) kk++;
                const int v = idx - kk * (kk + 1) / 2, u = kk - v, t = s - kk;
                // step down along z if t = u = 0, else along y if t = 0, else along x
                int uu = u, vv = v, kq, ax;
                if (t + u == 0) {
                    vv = v - 1;
                    kq = v;
                    ax = 2;
                } else if (t == 0) {
                    uu = u - 1;
                    kq = u;
                    ax = 1;
                } else {
                    kq = t;
                    ax = 0;
                }
                const int src1 = o1 + n * ne1 + r_in_level(uu, vv);
                int src2 = 0;
                if (kq > 1) src2 = o2 + n * ne2 + r_in_level(uu == u ? u : u - 2, vv == v ? v : v - 2);
                const int r0d = n == 0 ? r0_row(S, t, u) + v : kMmdNoR0;
                tab[lvl[s] + e] = int2{src1 | (src2 << 16), kq | (ax << 5) | (r0d << 7)};
            }
        }
    }
}

// Positions of work items in decreasing order of estimated work (buckets of a quarter
// octave; items of one bucket keep their order), for the kernels' dynamic queues.
static std::vector<int> order_by_cost(const std::vector<double> &cost)
{
    std::vector<int> key(cost.size());
    int kmax = 0;
    for (size_t i = 0; i < cost.size(); i++) {
        key[i] = cost[i] > 1.0 ? std::min(255, (int)(4.0 * std::log2(cost[i]))) : 0;
        kmax = std::max(kmax, key[i]);
    }
    std::vector<int> start(kmax + 2, 0), out(cost.size());
    for (int k : key) start[kmax - k + 1]++;
    for (int b = 1; b <= kmax + 1; b++) start[b] += start[b - 1];
    for (size_t i = 0; i < cost.size(); i++) out[start[kmax - key[i]]++] = (int)i;
    return out;
}

// Assembly classes and shared-memory layouts. A class is (la, lb, largest semilocal L, spin-orbit
// terms or not); the layout holds the task's RSH rows, both sides' omega tables, its radial
// table, the V rows of one potential (all rows when they fit in 6144 values) and W of the
// factored re-centring sum. W holds ncart(lb) x rows x (components + 1) values (the sums and the
// sums of absolute terms), rows chosen by the kernel so that nabB x rows x components fits in V;
// its size is set per launch group from the group's tasks.
static int fin_class_key(int la, int lb, int Lmax, bool so) { return ((la * 16 + lb) * 16 + Lmax) * 2 + (so ? 1 : 0); }

static int fin_default_nt(int la, int lb)
{
    const int w = n_abc(la) * n_abc(lb);
    return w < 1000 ? 128 : (w < 3000 ? 256 : 512);
}

static FinalSmem fin_layout(int lam, int n_omega, int n_q, int nabA, int nabB, int ncomp)
{
    FinalSmem fs{};
    fs.rsh_stride = 2 * lam + 1;
    fs.n_rsh = (lam + 1) * fs.rsh_stride;
    fs.n_omega = n_omega;
    fs.n_q = n_q;
    fs.n_v = std::min(6144, std::max(nabA * nabB * ncomp, 3 * std::max(nabA, nabB)));
    fs.n_v = std::max(fs.n_v, 3 * std::max(nabA, nabB));
    fs.n_w = 0;  // set per launch group
    return fs;
}

static FinalSmem fin_merge(const FinalSmem &x, const FinalSmem &y)
{
    FinalSmem m{};
    m.rsh_stride = std::max(x.rsh_stride, y.rsh_stride);
    m.n_rsh = std::max(x.n_rsh, y.n_rsh);
    m.n_omega = std::max(x.n_omega, y.n_omega);
    m.n_q = std::max(x.n_q, y.n_q);
    m.n_v = std::max(x.n_v, y.n_v);
    m.n_w = std::max(x.n_w, y.n_w);
    return m;
}

static size_t fin_smem_bytes(const FinalSmem &fs)
{
    return (size_t)(2 * fs.n_rsh + 2 * fs.n_omega + fs.n_q + fs.n_v + fs.n_w) * sizeof(double);
}

template <typename T>
T *at(void *base, size_t off)
{
    return (T *)((char *)base + off);
}

double host_gaussian_norm(int L, double a) { return std::pow(2 * a / kPi, 0.75) * std::pow(4 * a, 0.5 * L); }

double host_dfact(int n)
{
    double r = 1.0;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}

double host_factorial(int n)
{
    double r = 1.0;
    for (int k = 2; k <= n; k++) r *= k;
    return r;
}

// outercore_integrals.c:481-510: sqrt(2^(L+5/2) / Gamma(L+3/2)) alpha^(3/4+L/2)
double radial_gto_norm(int L, double alpha)
{
    const double g = host_dfact(2 * L + 1) * std::sqrt(kPi) / std::pow(2.0, L + 1);
    return std::sqrt(std::pow(2.0, L + 2.5) / g) * std::pow(alpha, 0.75 + L / 2.0);
}

// outercore_integrals.c:457-478
double one_centre_prim(int L, double a1, double a2, int n, double zeta)
{
    const double a = a1 + a2 + zeta;
    if (n % 2 == 0) {
        const int k = L + n / 2;
        return host_dfact(2 * k - 1) / (std::pow(2.0, k + 1) * std::pow(a, k)) * std::sqrt(kPi / a);
    }
    const int k = L + (n - 1) / 2;
    return host_factorial(k) / (2.0 * std::pow(a, k + 1));
}

// Entry offsets (l1 d2 dn + l2 dn + N) within a potential's (l1, l2, N) block that the
// type 2 and spin-orbit angular sums read (type2_integrals.c:169-184,
// spin_orbit_integrals.c:189-204): N = n1 + n2, n1 <= la, n2 <= lb, l1 in
// [max(L-n1, 0), L+n1] of the parity of L+n1, l2 likewise.
std::vector<uint16_t> used_entries(int L, int la, int lb)
{
    const int d2 = L + lb + 1, dn = la + lb + 1;
    std::vector<uint16_t> out;
    for (int l1 = 0; l1 <= L + la; l1++)
        for (int l2 = 0; l2 <= L + lb; l2++)
            for (int N = 0; N < dn; N++) {
                bool used = false;
                for (int n1 = std::max(0, N - lb); n1 <= std::min(la, N) && !used; n1++) {
                    const int n2 = N - n1;
                    used = l1 >= std::max(L - n1, 0) && l1 <= L + n1 && ((L + n1 - l1) & 1) == 0 &&
                           l2 >= std::max(L - n2, 0) && l2 <= L + n2 && ((L + n2 - l2) & 1) == 0;
                }
                if (used) out.push_back((uint16_t)((l1 * d2 + l2) * dn + N));
            }
    // screening order: the lanes of a warp take consecutive entries, and an entry's work grows
    // with l1 and with l2 (the Bessel sums of either side); tiles of 2 x 2 orders keep both
    // ranges narrow within a warp. The order only assigns entries to threads.
    auto key = [&](uint16_t e) {
        const int l1 = e / (d2 * dn), l2 = (e / dn) % d2;
        return ((l1 / 2) * 64 + l2 / 2) * 65536 + e;
    };
    std::stable_sort(out.begin(), out.end(), [&](uint16_t x, uint16_t y) { return key(x) < key(y); });
    return out;
}

struct PotView {
    int L, J;
    std::vector<int> pw;
    std::vector<double> c, a;
};
struct ShellView {
    int L;
    std::vector<double> c, a;
};

// outercore_integrals.c:397-450: delta = (U1 + U2)/2, Uk = <oc1| U_k |oc2> one-centre analytic
double delta_integral(const PotView &p1, const ShellView &s1, const PotView &p2, const ShellView &s2)
{
    if (p1.L != p2.L || p1.J != p2.J) return 0.0;
    auto U = [&](const PotView &p) {
        double sum = 0.0;
        const int L = p.L;
        for (size_t i = 0; i < s1.a.size(); i++) {
            const double Ni = radial_gto_norm(L, s1.a[i]);
            for (size_t j = 0; j < s2.a.size(); j++) {
                const double Nj = radial_gto_norm(L, s2.a[j]);
                const double f = Ni * Nj * s1.c[i] * s2.c[j];
                for (size_t k = 0; k < p.a.size(); k++) sum += f * p.c[k] * one_centre_prim(L, s1.a[i], s2.a[j], p.pw[k], p.a[k]);
            }
        }
        return sum;
    };
    return 0.5 * (U(p1) + U(p2));
}

int ensure_atab(DeviceState &st, int L, int l)
{
    const int key = L * (kMaxL + 2) + l;
    if (st.atab_off[key] >= 0) return 0;
    const int64_t sz = atab_size(L, l);
    const size_t need = (st.atab_used + sz) * sizeof(double);
    if (need > st.atab.cap) {
        void *old = st.atab.p;
        void *np = nullptr;
        size_t want = std::max(need * 2, (size_t)8 << 20);
        GRPP_CUDA(cudaMalloc(&np, want));
        if (old) {
            GRPP_CUDA(cudaMemcpyAsync(np, old, st.atab_used * sizeof(double), cudaMemcpyDeviceToDevice, st.stream));
            GRPP_CUDA(cudaStreamSynchronize(st.stream));
            cudaFree(old);
        }
        st.atab.p = np;
        st.atab.cap = want;
    }
    double *dst = (double *)st.atab.p + st.atab_used;
    const int threads = 256;
    const int blocks = (int)std::min<int64_t>((sz + threads - 1) / threads, 4096);
    GRPP_CUDA(ang_launch_atab(std::max(blocks, 1), threads, st.stream, L, l, dst));
    st.atab_off[key] = (int64_t)st.atab_used;
    st.atab_used += sz;
    st.atab_dirty = true;
    return 0;
}

}  // namespace

// One launch of the assembly kernel: the tasks order[first .. first+count) of one block size, with
// a shared-memory layout sized for the largest of them. Small tasks in a group of their own get
// small layouts and many blocks per SM; the block size per assembly class comes from the
// autotuner's table (libgrpp_b200_autotune_assembly) or the default rule.
struct FinGroup {
    int nt = 128;
    int first = 0, count = 0;
    int key = -1;  // assembly class when the groups are one per class (autotuning), else -1
    FinalSmem fs{};
    size_t smem = 0;
    int blocks = 0;
    float ms = 0.f;
};

struct Plan {
    DeviceState *st = nullptr;
    int set = 0;  // buffer set, events and status words of the device state it uses
    RunOptions opt;
    int64_t n_tasks = 0, out_tot = 0, n_radial = 0, n_mmd = 0, n_entries = 0, h2d_bytes = 0, scratch_bytes = 0;
    DevBuf in, scratch, out;
    double *outs[4] = {nullptr, nullptr, nullptr, nullptr};
    int *status = nullptr;
    unsigned long long *counters = nullptr;  // kRadCntNum slots inside the status area
    int8_t *stop_level = nullptr, *pred_level = nullptr;  // per radial item
    int *order = nullptr, *lm_ctl = nullptr;               // learned mode: item order; n_order, queue, cursor[9]
    MmdArgs mmd;
    int mmd_blocks = 0, mmd_threads = 128, mmd_kpl = 32;
    size_t mmd_smem = 0;
    OcProjArgs ocp;
    int ocp_blocks = 0;
    RadialArgs rad;
    int rad_blocks = 0, scr_blocks = 0, scru_blocks = 0;
    size_t scru_smem = 0;
    double *wu = nullptr;  // w U_p(r) table (scratch), filled by wu_table_kernel before the walk
    int wu_grpps = 0, wu_blocks = 0;
    double *ftab = nullptr;  // F_l(r) tables per (shell, centre) pair (scratch), ftab_kernel
    int ft_blocks = 0;
    size_t ft_smem = 0;
    double *omtab = nullptr;  // omega tables per (shell, centre) pair (scratch), omega_tab_kernel
    const int *om_shell = nullptr, *om_centre = nullptr;
    int om_pairs = 0, om_blocks = 0;
    size_t om_smem = 0;
    size_t rad_smem = 0;
    FinalArgs fin;
    FinalSmem fin_smem_layout;  // batch-wide layout (omega tables)
    std::vector<FinGroup> fin_groups;
    int *fin_queue = nullptr;   // one counter per group
    bool time_groups = false;   // record an event between the assembly launches
    RunStats stats;
    bool count_ops = false;  // run the type 1 kernel's counting instantiation
};

int64_t batch_output_size(const libgrpp_b200_batch_t *b)
{
    int64_t n = 0;
    for (int64_t t = 0; t < b->n_tasks; t++) n += (int64_t)ncart(b->shell_L[b->task_a[t]]) * ncart(b->shell_L[b->task_b[t]]);
    return n;
}

#define CHECK_INPUT(cond, msg)                               \
    do {                                                     \
        if (!(cond)) {                                       \
            set_error(LIBGRPP_B200_ERR_INVALID, (msg));      \
            return LIBGRPP_B200_ERR_INVALID;                 \
        }                                                    \
    } while (0)

// Host preprocessing, upload and kernel arguments of one batch. With own_buffers the
// plan allocates its device memory (kept until plan_destroy); otherwise it borrows the
// device state's buffers and is valid until the next batch on that device.
int plan_build(DeviceState &st, const libgrpp_b200_batch_t *b, const RunOptions &opt, bool own_buffers, Plan &P,
               int set = 0)
{
    int rc = 0;
    cudaStream_t s = st.stream;
    const int64_t nt = b->n_tasks;
    P.st = &st;
    P.set = set;
    P.n_tasks = nt;
    P.opt = opt;
    if (nt == 0) return 0;

    // ---------------------------------------------------------------- validation
    CHECK_INPUT(b->n_shells > 0 && b->n_centres > 0 && b->n_grpps > 0, "empty batch description");
    for (int i = 0; i < b->n_shells; i++) {
        CHECK_INPUT(b->shell_L[i] >= 0 && b->shell_L[i] <= kMaxL, "shell angular momentum outside 0..10");
        CHECK_INPUT(b->shell_nprim[i] >= 0 && b->shell_nprim[i] <= kRadMaxPrims, "more than 64 primitives in a shell");
    }
    for (int p = 0; p < b->n_pots; p++) {
        CHECK_INPUT(b->pot_L[p] >= 0 && b->pot_L[p] <= kMaxL, "potential angular momentum outside 0..10");
        for (int k = 0; k < b->pot_nprim[p]; k++) {
            const int n = b->pot_powers[b->pot_prim_off[p] + k];
            CHECK_INPUT(n >= 0 && n <= 2, "potential power n must be 0, 1 or 2");
        }
    }
    for (int64_t t = 0; t < nt; t++) {
        CHECK_INPUT(b->task_a[t] >= 0 && b->task_a[t] < b->n_shells && b->task_b[t] >= 0 && b->task_b[t] < b->n_shells &&
                        b->task_c[t] >= 0 && b->task_c[t] < b->n_centres,
                    "task index out of range");
    }
    for (int c = 0; c < b->n_centres; c++) CHECK_INPUT(b->centre_grpp[c] >= 0 && b->centre_grpp[c] < b->n_grpps, "centre GRPP index out of range");

    // ---------------------------------------------------------------- shells
    const int ns = b->n_shells;
    std::vector<int> sh_L(b->shell_L, b->shell_L + ns), sh_np(b->shell_nprim, b->shell_nprim + ns),
        sh_po(b->shell_prim_off, b->shell_prim_off + ns), sh_co(ns);
    int total_prims = 0;
    for (int i = 0; i < ns; i++) total_prims = std::max(total_prims, sh_po[i] + sh_np[i]);
    std::vector<double> pc(b->prim_coef, b->prim_coef + total_prims), pa(b->prim_alpha, b->prim_alpha + total_prims);
    std::vector<double> sh_or(b->shell_origin, b->shell_origin + 3 * ns);
    std::vector<int8_t> cart;
    for (int i = 0; i < ns; i++) {
        sh_co[i] = (int)(cart.size() / 3);
        const int nc = ncart(sh_L[i]);
        for (int q = 0; q < 3 * nc; q++) {
            const int v = b->cart_list[3 * b->shell_cart_off[i] + q];
            CHECK_INPUT(v >= 0 && v <= sh_L[i], "invalid Cartesian component list");
            cart.push_back((int8_t)v);
        }
    }
    // radial-path primitives: shrunk and normalised (radial_type2_integral.c:164-172)
    std::vector<int> rp_off(ns), rp_n(ns);
    std::vector<double> rp_c, rp_a;
    for (int i = 0; i < ns; i++) {
        rp_off[i] = (int)rp_c.size();
        for (int k = 0; k < sh_np[i]; k++) {
            const double c = pc[sh_po[i] + k], a = pa[sh_po[i] + k];
            if (std::fabs(c) > kZeroThresh) {
                rp_c.push_back(c * host_gaussian_norm(sh_L[i], a));
                rp_a.push_back(a);
            }
        }
        rp_n[i] = (int)rp_c.size() - rp_off[i];
    }

    // ---------------------------------------------------------------- potentials (|c| < 1e-14 dropped, potential.c:31-42)
    const int np = b->n_pots;
    std::vector<int> p_L(np), p_n(np), p_off(np), p_pw;
    std::vector<double> p_c, p_a;
    std::vector<PotView> pview(np);
    for (int p = 0; p < np; p++) {
        p_L[p] = b->pot_L[p];
        p_off[p] = (int)p_c.size();
        pview[p].L = b->pot_L[p];
        pview[p].J = b->pot_J[p];
        for (int k = 0; k < b->pot_nprim[p]; k++) {
            const int o = b->pot_prim_off[p] + k;
            if (std::fabs(b->pot_coef[o]) < kZeroThresh) continue;
            p_pw.push_back(b->pot_powers[o]);
            p_c.push_back(b->pot_coef[o]);
            p_a.push_back(b->pot_alpha[o]);
            pview[p].pw.push_back(b->pot_powers[o]);
            pview[p].c.push_back(b->pot_coef[o]);
            pview[p].a.push_back(b->pot_alpha[o]);
        }
        p_n[p] = (int)p_c.size() - p_off[p];
    }

    // ---------------------------------------------------------------- GRPP operators
    const int ng = b->n_grpps;
    std::vector<int> g_sl_off(ng), g_sl_n(ng), g_n_arep(ng), sl_pot, g_oc_off(ng), g_n_oc(ng), oc_L, oc_J, oc_pot,
        oc_shell, g_delta_off(ng);
    std::vector<double> deltas;
    for (int g = 0; g < ng; g++) {
        g_sl_off[g] = (int)sl_pot.size();
        for (int i = 0; i < b->grpp_n_arep[g]; i++) sl_pot.push_back(b->grpp_pot_list[b->grpp_arep_off[g] + i]);
        for (int i = 0; i < b->grpp_n_so[g]; i++) sl_pot.push_back(b->grpp_pot_list[b->grpp_so_off[g] + i]);
        g_n_arep[g] = b->grpp_n_arep[g];
        g_sl_n[g] = (int)sl_pot.size() - g_sl_off[g];
        CHECK_INPUT(g_sl_n[g] <= kRadMaxPots, "more than 24 semilocal potentials in one GRPP");
        int nterm = 0;
        for (int i = g_sl_off[g]; i < g_sl_off[g] + g_sl_n[g]; i++) nterm += p_n[sl_pot[i]];
        CHECK_INPUT(nterm <= kRadMaxTerms, "more than 256 semilocal potential terms in one GRPP");
        g_oc_off[g] = (int)oc_L.size();
        g_n_oc[g] = b->grpp_n_oc[g];
        CHECK_INPUT(g_n_oc[g] <= kFinMaxOc, "more than 32 outercore shells in one GRPP");
        for (int i = 0; i < g_n_oc[g]; i++) {
            const int k = b->grpp_oc_off[g] + i;
            const int pp = b->grpp_oc_pot[k], so = b->grpp_oc_shell[k];
            CHECK_INPUT(sh_L[so] == p_L[pp], "outercore shell and potential differ in L");
            oc_L.push_back(sh_L[so]);
            oc_J.push_back(b->pot_J[pp]);
            oc_pot.push_back(pp);
            oc_shell.push_back(so);
        }
        g_delta_off[g] = (int)deltas.size();
        const int n = g_n_oc[g];
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                const int ki = g_oc_off[g] + i, kj = g_oc_off[g] + j;
                ShellView si{sh_L[oc_shell[ki]], {}, {}}, sj{sh_L[oc_shell[kj]], {}, {}};
                for (int q = 0; q < sh_np[oc_shell[ki]]; q++) {
                    si.c.push_back(pc[sh_po[oc_shell[ki]] + q]);
                    si.a.push_back(pa[sh_po[oc_shell[ki]] + q]);
                }
                for (int q = 0; q < sh_np[oc_shell[kj]]; q++) {
                    sj.c.push_back(pc[sh_po[oc_shell[kj]] + q]);
                    sj.a.push_back(pa[sh_po[oc_shell[kj]] + q]);
                }
                deltas.push_back(delta_integral(pview[oc_pot[ki]], si, pview[oc_pot[kj]], sj));
            }
    }

    // ---------------------------------------------------------------- tasks and work lists
    std::vector<int> ta(b->task_a, b->task_a + nt), tb(b->task_b, b->task_b + nt), tc(b->task_c, b->task_c + nt);
    std::vector<int64_t> out_off(nt + 1), q_off(nt, -1);
    std::vector<uint8_t> has_ul(nt, 0);
    std::vector<int> proj_a(nt, -1), proj_b(nt, -1);
    std::vector<MmdItem> items;
    std::vector<int> rad_task;
    std::vector<int64_t> rad_qoff, rad_uoff;
    // (shell, centre) pairs of the radial items, for the F_l(r) tables (ftab_kernel)
    // pair index per (shell, centre): a flat array when it is small next to the chunk (filling
    // it costs n_shells x n_centres per chunk), else a hash map
    const int64_t n_sc = (int64_t)b->n_shells * b->n_centres;
    std::vector<int> fpair_flat(n_sc <= std::max<int64_t>(8 * nt, 4096) ? n_sc : 0, -1);
    std::unordered_map<int64_t, int> fpair_of;
    std::vector<int> fp_shell, fp_centre, fp_lmax, item_fa, item_fb;
    std::vector<int> task_fpa(nt, -1), task_fpb(nt, -1);
    auto fpair = [&](int shell, int centre, int lmax) {
        const int64_t key = (int64_t)shell * b->n_centres + centre;
        int idx = -1;
        if (!fpair_flat.empty()) {
            idx = fpair_flat[key];
        } else {
            const auto f = fpair_of.find(key);
            if (f != fpair_of.end()) idx = f->second;
        }
        if (idx < 0) {
            idx = (int)fp_shell.size();
            if (!fpair_flat.empty()) fpair_flat[key] = idx;
            else fpair_of[key] = idx;
            fp_shell.push_back(shell);
            fp_centre.push_back(centre);
            fp_lmax.push_back(lmax);
        } else {
            fp_lmax[idx] = std::max(fp_lmax[idx], lmax);
        }
        return idx;
    };
    int64_t qtot = 0, utot = 0, rad_list_max = 0;
    // screening runs: long runs of one (task, potential) to the unit kernel, short ones (and
    // one-centre tasks) to the flat kernel
    std::vector<ScrUnit> scr_big, scr_small;
    std::vector<int64_t> su_off(1, 0);
    int scr_lw = 2;
    std::vector<int2> ucls((kMaxL + 1) * (kMaxL + 1) * (kMaxL + 1), int2{0, 0});
    std::vector<uint8_t> ucls_set(ucls.size(), 0);
    std::vector<uint16_t> ulist;
    out_off[0] = 0;
    int mmd_lmax = 0, mmd_smax = 0;
    int rad_l1 = 0, rad_l2 = 0, rad_dn = 1, rad_npot = 0;
    int fin_lam = 0, fin_nq = 1;
    std::map<std::pair<int, int>, int> proj_map;
    std::vector<std::pair<int, int>> projs;
    std::vector<std::pair<int, int>> atab_need;
    std::vector<uint8_t> atab_flag((kMaxL + 1) * (kMaxL + 1), 0);  // (L, l) pairs seen
    for (int64_t t = 0; t < nt; t++) {
        const int A = ta[t], B = tb[t], C = tc[t], g = b->centre_grpp[C];
        const int la = sh_L[A], lb = sh_L[B];
        CHECK_INPUT(sh_np[A] >= 1 && sh_np[B] >= 1, "a shell of a task has no primitives");
        CHECK_INPUT(ncart(la) * ncart(lb) <= kFinMaxPairs, "shell pair block larger than 1024 Cartesian pairs");
        out_off[t + 1] = out_off[t] + (int64_t)ncart(la) * ncart(lb);
        if (b->grpp_UL[g] >= 0 && p_n[b->grpp_UL[g]] > 0) {
            has_ul[t] = 1;
            MmdItem it{A, B, 0, C, b->grpp_UL[g], 0, out_off[t]};
            items.push_back(it);
            mmd_lmax = std::max(mmd_lmax, std::max(la, lb));
            mmd_smax = std::max(mmd_smax, la + lb);
        }
        if (g_sl_n[g] > 0) {
            q_off[t] = qtot;
            rad_task.push_back((int)t);
            rad_qoff.push_back(qtot);
            rad_uoff.push_back(utot);
            int e = 0, Lmx = 0;
            int64_t item_used = 0;
            double CA2 = 0.0, CB2 = 0.0;
            for (int d = 0; d < 3; d++) {
                const double u = b->centre_origin[3 * C + d] - b->shell_origin[3 * A + d];
                const double v = b->centre_origin[3 * C + d] - b->shell_origin[3 * B + d];
                CA2 += u * u;
                CB2 += v * v;
            }
            const bool one_centre = CA2 < 1e-14 && CB2 < 1e-14;
            const int item = (int)rad_task.size() - 1;
            for (int i = 0; i < g_sl_n[g]; i++) {
                const int pot = sl_pot[g_sl_off[g] + i];
                const int L = p_L[pot];
                Lmx = std::max(Lmx, L);
                const int pe = e;
                e += (L + la + 1) * (L + lb + 1) * (la + lb + 1);
                const int key = (L * (kMaxL + 1) + la) * (kMaxL + 1) + lb;
                if (!ucls_set[key]) {
                    const std::vector<uint16_t> u = used_entries(L, la, lb);
                    ucls[key] = int2{(int)ulist.size(), (int)u.size()};
                    ulist.insert(ulist.end(), u.begin(), u.end());
                    ucls_set[key] = 1;
                }
                const int ne = ucls[key].y;
                if (one_centre || ne < kScrUnitMin) {
                    if (ne > 0) {
                        scr_small.push_back(ScrUnit{item, pot, pe, ucls[key].x, ne});
                        su_off.push_back(su_off.back() + ne);
                    }
                } else {
                    for (int o = 0; o < ne; o += kScrUnitThreads)
                        scr_big.push_back(ScrUnit{item, pot, pe, ucls[key].x + o, std::min(kScrUnitThreads, ne - o)});
                    scr_lw = std::max(scr_lw, L + std::max(la, lb) + 1);
                }
                utot += ucls[key].y;
                item_used += ucls[key].y;
                rad_l1 = std::max(rad_l1, L + la);
                rad_l2 = std::max(rad_l2, L + lb);
                fin_lam = std::max(fin_lam, L + std::max(la, lb));
                fin_nq = std::max(fin_nq, (L + la + 1) * (L + lb + 1) * (la + lb + 1));
                atab_flag[L * (kMaxL + 1) + la] = 1;
                atab_flag[L * (kMaxL + 1) + lb] = 1;
            }
            CHECK_INPUT(e <= kRadMaxEntries, "radial table larger than 16384 entries for one task");
            item_fa.push_back(fpair(A, C, Lmx + la));
            item_fb.push_back(fpair(B, C, Lmx + lb));
            task_fpa[t] = item_fa.back();
            task_fpb[t] = item_fb.back();
            CHECK_INPUT(std::max(rad_l1, rad_l2) <= kRadMaxLam && la + lb + 1 <= kRadMaxN, "angular momentum too high for the radial path");
            qtot += e;
            rad_list_max = std::max(rad_list_max, item_used);
            rad_dn = std::max(rad_dn, la + lb + 1);
            rad_npot = std::max(rad_npot, g_sl_n[g]);
        }
        if (g_n_oc[g] > 0) {
            for (int side = 0; side < 2; side++) {
                const int S = side ? B : A;
                auto key = std::make_pair(S, C);
                auto itp = proj_map.find(key);
                int idx;
                if (itp == proj_map.end()) {
                    idx = (int)projs.size();
                    proj_map[key] = idx;
                    projs.push_back(key);
                } else {
                    idx = itp->second;
                }
                (side ? proj_b : proj_a)[t] = idx;
            }
        }
    }
    // long screening runs, costliest first (entries x primitive triples), so the static
    // round-robin over blocks ends evenly
    {
        auto cost = [&](const ScrUnit &u) {
            const int t = rad_task[u.item];
            return (int64_t)u.ne * rp_n[ta[t]] * rp_n[tb[t]] * p_n[u.pot];
        };
        std::stable_sort(scr_big.begin(), scr_big.end(), [&](const ScrUnit &x, const ScrUnit &y) { return cost(x) > cost(y); });
    }
    // outercore projection blocks
    std::vector<int> blk_shell, blk_oc;
    std::vector<int64_t> blk_cart_off, blk_sph_off, proj_off(projs.size() + 1, 0);
    int64_t cart_tot = 0, sph_tot = 0;
    for (size_t pi = 0; pi < projs.size(); pi++) {
        const int S = projs[pi].first, C = projs[pi].second, g = b->centre_grpp[C];
        proj_off[pi] = sph_tot;
        for (int k = 0; k < g_n_oc[g]; k++) {
            const int ko = g_oc_off[g] + k, osh = oc_shell[ko], L = oc_L[ko];
            blk_shell.push_back(S);
            blk_oc.push_back(osh);
            blk_cart_off.push_back(cart_tot);
            blk_sph_off.push_back(sph_tot);
            items.push_back(MmdItem{S, osh, 1, C, oc_pot[ko], 1, cart_tot});
            items.push_back(MmdItem{S, osh, 1, C, -1, 2, cart_tot});
            mmd_lmax = std::max(mmd_lmax, std::max(sh_L[S], L));
            mmd_smax = std::max(mmd_smax, sh_L[S] + L);
            cart_tot += (int64_t)ncart(sh_L[S]) * ncart(L);
            sph_tot += (int64_t)ncart(sh_L[S]) * (2 * L + 1);
        }
    }
    proj_off[projs.size()] = sph_tot;
    const int64_t out_tot = out_off[nt];

    // Cartesian pair schedules of the type 1 items, one per (bra, ket) table class
    const int mmd_kpl = ncart(mmd_lmax) * ncart(mmd_lmax) <= 256 ? 8 : 32;
    std::vector<uint16_t> mmd_sched;
    {
        std::map<std::vector<int8_t>, int> tab_id;  // a shell's Cartesian table -> class
        std::vector<int> sh_tab(ns);
        for (int i = 0; i < ns; i++) {
            const std::vector<int8_t> tab(cart.begin() + 3 * sh_co[i], cart.begin() + 3 * (sh_co[i] + ncart(sh_L[i])));
            auto ins = tab_id.insert({tab, (int)tab_id.size()});
            sh_tab[i] = ins.first->second;
        }
        const int ntab = (int)tab_id.size();
        std::vector<std::pair<int, int>> sched_of((size_t)ntab * ntab, {-1, 0});  // (bra, ket) class -> (offset, rows)
        for (auto &it : items) {
            const int nA = ncart(sh_L[it.bra]), nB = ncart(sh_L[it.ket]);
            CHECK_INPUT(nA * nB <= 32 * mmd_kpl, "type 1 block larger than one pass of the pair schedule");
            std::pair<int, int> &f = sched_of[(size_t)sh_tab[it.bra] * ntab + sh_tab[it.ket]];
            if (f.first < 0) {
                const int off = (int)mmd_sched.size();
                const int rows = mmd_pair_schedule(cart.data() + 3 * sh_co[it.bra], nA, cart.data() + 3 * sh_co[it.ket],
                                                   nB, mmd_kpl, mmd_sched);
                f = {off, rows};
            }
            it.sched = f.first;
            it.sched_rows = f.second;
        }
    }
    // estimated work per type 1 item: primitive triples x (Hermite + R entries + contraction terms)
    std::vector<int> mmd_order;
    {
        std::vector<double> cost(items.size());
        for (size_t q = 0; q < items.size(); q++) {
            const MmdItem &it = items[q];
            const int la = sh_L[it.bra], lb = sh_L[it.ket], S = la + lb;
            const double np2 = (double)sh_np[it.bra] * sh_np[it.ket], pairs = (double)ncart(la) * ncart(lb);
            if (it.pot < 0) cost[q] = np2 * (pairs + 10.0);
            else
                cost[q] = np2 * p_n[it.pot] *
                          (mmd_e_count(la, lb) + mmd_r_size(S) + pairs * (S + 3.0) * (S + 3.0) * (S + 3.0) / 27.0);
        }
        mmd_order = order_by_cost(cost);
    }

    // Assembly launch groups. Per task: its class, the block size for the class (the caller's,
    // the autotuner's table, or the default rule) and the shared memory its tables need. Tasks of
    // one block size and one shared-memory tier form a group (one group per class when
    // autotuning); within a group the queue takes the largest estimated work first: per
    // semilocal potential, the V table and the re-centring sums of its Cartesian pairs.
    std::vector<int> fin_order;
    std::vector<FinGroup> fin_groups;
    {
        std::vector<double> cost(nt);
        std::map<int, int> gidx;
        std::vector<std::vector<int>> members;
        for (int64_t t = 0; t < nt; t++) {
            const int la = sh_L[ta[t]], lb = sh_L[tb[t]], g = b->centre_grpp[tc[t]];
            cost[t] = 1.0 + (double)g_sl_n[g] * ((double)n_abc(la) * n_abc(lb) + 4.0 * ncart(la) * ncart(lb));
            int lam = 0, nom = 1, nq = 1, Lmx = 0;
            for (int i = 0; i < g_sl_n[g]; i++) {
                const int L = p_L[sl_pot[g_sl_off[g] + i]];
                Lmx = std::max(Lmx, L);
                lam = std::max(lam, L + std::max(la, lb));
                nom = std::max(nom, std::max(n_abc(la) * lam_slots(L, la), n_abc(lb) * lam_slots(L, lb)) * (2 * L + 1));
                nq = std::max(nq, (L + la + 1) * (L + lb + 1) * (la + lb + 1));
            }
            const bool so = b->grpp_n_so[g] > 0;
            const int cls = fin_class_key(la, lb, Lmx, so);
            int ntb = opt.fin_nt;
            if (ntb == 0) {
                auto it = st.fin_tune.find(cls);
                ntb = it != st.fin_tune.end() ? it->second : fin_default_nt(la, lb);
            }
            CHECK_INPUT(ntb == 128 || ntb == 256 || ntb == 512, "assembly block size must be 128, 256 or 512");
            const FinalSmem fs = fin_layout(lam, nom, nq, n_abc(la), n_abc(lb), so ? 3 : 1);
            const size_t bytes = fin_smem_bytes(fs);
            const int tier = bytes <= 32 * 1024 ? 0 : (bytes <= 96 * 1024 ? 1 : 2);
            const int key = opt.fin_by_class ? cls * 8 + ntb / 128 : ntb * 4 + tier;
            auto it = gidx.find(key);
            int gi;
            if (it == gidx.end()) {
                gi = (int)fin_groups.size();
                gidx[key] = gi;
                FinGroup G;
                G.nt = ntb;
                G.key = opt.fin_by_class ? cls : -1;
                G.fs = fs;
                fin_groups.push_back(G);
                members.emplace_back();
            } else {
                gi = it->second;
                fin_groups[gi].fs = fin_merge(fin_groups[gi].fs, fs);
            }
            members[gi].push_back((int)t);
        }
        for (size_t gi = 0; gi < fin_groups.size(); gi++) {
            auto &m = members[gi];
            std::stable_sort(m.begin(), m.end(), [&](int x, int y) { return cost[x] > cost[y]; });
            fin_groups[gi].first = (int)fin_order.size();
            fin_groups[gi].count = (int)m.size();
            fin_order.insert(fin_order.end(), m.begin(), m.end());
            FinalSmem &fs = fin_groups[gi].fs;
            // W of the factored re-centring sum: ncart(lb) x rows x (components + 1) values per
            // potential, rows as the kernel takes them from the group's V size
            int need = 0;
            for (int t : m) {
                const int la = sh_L[ta[t]], lb = sh_L[tb[t]];
                const bool so = b->grpp_n_so[b->centre_grpp[tc[t]]] > 0;
                for (int ncomp = 1; ncomp <= (so ? 3 : 1); ncomp += 2) {
                    const int rows = std::max(1, std::min(n_abc(la), fs.n_v / (n_abc(lb) * ncomp)));
                    need = std::max(need, ncart(lb) * rows * (ncomp + 1));
                }
            }
            fs.n_w = need;
            if (fin_smem_bytes(fs) > kFinSmemMax) fs.n_w = 0;  // term-by-term re-centring only
            CHECK_INPUT(fin_smem_bytes(fs) <= kFinSmemMax, "assembly tables of this batch exceed the shared memory of one block");
            fin_groups[gi].smem = fin_smem_bytes(fs);
        }
    }
    std::vector<int> mmd_etab, mmd_etab_off, mmd_rtab_off;
    std::vector<int2> mmd_rtab;
    mmd_update_tables(mmd_lmax, mmd_smax, mmd_etab, mmd_etab_off, mmd_rtab, mmd_rtab_off);

    // F_l(r) tables per (shell, centre) pair: (lmax + 1) rows of grid points each, when they
    // stay below 8 GiB
    std::vector<int64_t> fp_off(fp_shell.size() + 1, 0);
    for (size_t k = 0; k < fp_shell.size(); k++) fp_off[k + 1] = fp_off[k] + (int64_t)(fp_lmax[k] + 1) * kRadGridPts;
    int64_t f_words = rad_task.empty() ? 0 : fp_off.back();
    if (f_words * (int64_t)sizeof(double) > (int64_t(8) << 30)) f_words = 0;
    // omega tables per (shell, centre) pair (omega_tab_kernel): per semilocal potential of the
    // centre's GRPP, n_abc(l) x slots x (2L+1) values; below 2 GiB
    std::vector<int64_t> om_off(fp_shell.size() + 1, 0);
    for (size_t k = 0; k < fp_shell.size(); k++) {
        const int l = sh_L[fp_shell[k]], g = b->centre_grpp[fp_centre[k]];
        int64_t w = 0;
        for (int i = 0; i < g_sl_n[g]; i++) {
            const int L = p_L[sl_pot[g_sl_off[g] + i]];
            w += (int64_t)n_abc(l) * lam_slots(L, l) * (2 * L + 1);
        }
        om_off[k + 1] = om_off[k] + w;
    }
    int64_t om_words = rad_task.empty() ? 0 : om_off.back();
    if (om_words * (int64_t)sizeof(double) > (int64_t(2) << 30)) om_words = 0;

    // angular tensors
    for (int L = 0; L <= kMaxL; L++)
        for (int l = 0; l <= kMaxL; l++)
            if (atab_flag[L * (kMaxL + 1) + l]) atab_need.push_back({L, l});
    for (auto &lp : atab_need) {
        rc = ensure_atab(st, lp.first, lp.second);
        if (rc) return rc;
    }
    if (st.atab_dirty) {  // offsets of newly built tables (existing offsets never change)
        GRPP_CUDA(st.atab_off_dev.ensure(st.atab_off.size() * sizeof(int64_t)));
        GRPP_CUDA(cudaMemcpyAsync(st.atab_off_dev.p, st.atab_off.data(), st.atab_off.size() * sizeof(int64_t),
                                  cudaMemcpyHostToDevice, s));
        GRPP_CUDA(cudaStreamSynchronize(s));
        st.atab_dirty = false;
    }

    // ---------------------------------------------------------------- upload
    std::vector<int> sh_po_v(sh_po), cart_off_v(sh_co);
    std::vector<double> c_or(b->centre_origin, b->centre_origin + 3 * b->n_centres);
    std::vector<int> c_g(b->centre_grpp, b->centre_grpp + b->n_centres);
    Packer pk;
    const size_t o_shL = pk.add(sh_L), o_shnp = pk.add(sh_np), o_shpo = pk.add(sh_po_v), o_shco = pk.add(cart_off_v);
    const size_t o_pc = pk.add(pc), o_pa = pk.add(pa), o_sor = pk.add(sh_or), o_cart = pk.add(cart);
    const size_t o_rpo = pk.add(rp_off), o_rpn = pk.add(rp_n), o_rpc = pk.add(rp_c), o_rpa = pk.add(rp_a);
    const size_t o_pL = pk.add(p_L), o_pn = pk.add(p_n), o_poff = pk.add(p_off), o_ppw = pk.add(p_pw), o_pcoef = pk.add(p_c),
                 o_palpha = pk.add(p_a);
    const size_t o_gslo = pk.add(g_sl_off), o_gsln = pk.add(g_sl_n), o_gnar = pk.add(g_n_arep), o_slp = pk.add(sl_pot);
    const size_t o_goco = pk.add(g_oc_off), o_gnoc = pk.add(g_n_oc), o_ocL = pk.add(oc_L), o_ocJ = pk.add(oc_J),
                 o_gdo = pk.add(g_delta_off), o_del = pk.add(deltas);
    const size_t o_cor = pk.add(c_or), o_cg = pk.add(c_g);
    const size_t o_ta = pk.add(ta), o_tb = pk.add(tb), o_tc = pk.add(tc), o_too = pk.add(out_off), o_thul = pk.add(has_ul),
                 o_tqo = pk.add(q_off), o_tpa = pk.add(proj_a), o_tpb = pk.add(proj_b);
    const size_t o_items = pk.add(items), o_rt = pk.add(rad_task), o_rq = pk.add(rad_qoff), o_ru = pk.add(rad_uoff),
                 o_ucls = pk.add(ucls), o_ulist = pk.add(ulist), o_sbig = pk.add(scr_big), o_ssmall = pk.add(scr_small),
                 o_suo = pk.add(su_off);
    const size_t o_bs = pk.add(blk_shell), o_bo = pk.add(blk_oc), o_bco = pk.add(blk_cart_off), o_bso = pk.add(blk_sph_off),
                 o_poffp = pk.add(proj_off), o_msch = pk.add(mmd_sched);
    const size_t o_fps = pk.add(fp_shell), o_fpc = pk.add(fp_centre), o_fpl = pk.add(fp_lmax), o_fpo = pk.add(fp_off),
                 o_ifa = pk.add(item_fa), o_ifb = pk.add(item_fb), o_omo = pk.add(om_off), o_tfa = pk.add(task_fpa),
                 o_tfb = pk.add(task_fpb);
    const size_t o_met = pk.add(mmd_etab), o_meto = pk.add(mmd_etab_off), o_mrt = pk.add(mmd_rtab),
                 o_mrto = pk.add(mmd_rtab_off), o_mord = pk.add(mmd_order), o_ford = pk.add(fin_order);
    std::vector<int8_t> stop_dummy;
    DevBuf *bin = own_buffers ? &P.in : &st.in[set], *bscr = own_buffers ? &P.scratch : &st.scratch[set],
           *bout = own_buffers ? &P.out : &st.out[set];
    GRPP_CUDA(bin->ensure(pk.buf.size()));
    // through the set's page-locked staging buffer, once its previous upload has finished
    GRPP_CUDA(cudaEventSynchronize(st.uploaded[set]));
    GRPP_CUDA(st.stage[set].ensure(pk.buf.size()));
    memcpy(st.stage[set].p, pk.buf.data(), pk.buf.size());
    GRPP_CUDA(cudaMemcpyAsync(bin->p, st.stage[set].p, pk.buf.size(), cudaMemcpyHostToDevice, s));
    GRPP_CUDA(cudaEventRecord(st.uploaded[set], s));
    P.h2d_bytes = (int64_t)pk.buf.size();
    void *ib = bin->p;

    // scratch: Q, S_prev, scr | S_cart, U_cart | S_sph, U_sph | status ; outputs: 4 x out_tot
    const int64_t qn = std::max<int64_t>(qtot, 1), cn = std::max<int64_t>(cart_tot, 1), sn = std::max<int64_t>(sph_tot, 1);
    const int64_t nrad = std::max<int64_t>((int64_t)rad_task.size(), 1);
    const int64_t flag_words = (qn + nrad + 2 * 8) / 8 + 1;  // entry flags + per-task walk flags, in doubles
    // per radial item: stop level, predicted level (int8), order (int); learned-mode control words
    const int64_t lm_words = (2 * nrad + 4 * nrad + 16 * 4) / 8 + 4;
    // table of w U_p(r) per GRPP, semilocal potential slot and grid point (wu_table_kernel),
    // when the batch walks a grid and the table stays below 256 MiB
    int wu_npot = 0;
    for (int g = 0; g < ng; g++) wu_npot = std::max(wu_npot, g_sl_n[g]);
    int64_t wu_words = rad_task.empty() ? 0 : (int64_t)ng * wu_npot * kRadGridPts;
    if (wu_words * (int64_t)sizeof(double) > (int64_t(256) << 20)) wu_words = 0;
    const size_t scratch_bytes =
        (size_t)(3 * qn + 2 * cn + 2 * sn + 16 + 16 + flag_words + lm_words + wu_words + f_words + om_words) *
        sizeof(double);
    GRPP_CUDA(bscr->ensure(scratch_bytes));
    GRPP_CUDA(bout->ensure((size_t)4 * std::max<int64_t>(out_tot, 1) * sizeof(double)));
    P.scratch_bytes = (int64_t)scratch_bytes;
    double *Qd = (double *)bscr->p, *Spd = Qd + qn, *SCd = Spd + qn, *Scd = SCd + qn, *Ucd = Scd + cn, *Ssd = Ucd + cn,
           *Usd = Ssd + sn;
    int *statusd = (int *)(Usd + sn);
    uint8_t *eflagd = (uint8_t *)(Usd + sn + 32);
    uint8_t *walkd = eflagd + qn;
    int8_t *stopd = (int8_t *)(Usd + sn + 32 + flag_words);
    int8_t *predd = stopd + nrad;
    int *orderd = (int *)(((uintptr_t)(predd + nrad) + 15) & ~(uintptr_t)15);
    int *lmctld = orderd + nrad;
    double *wud = wu_words > 0 ? (double *)bscr->p + (3 * qn + 2 * cn + 2 * sn + 16 + 16 + flag_words + lm_words) : nullptr;
    double *ftd = f_words > 0 ? (double *)bscr->p + (3 * qn + 2 * cn + 2 * sn + 16 + 16 + flag_words + lm_words + wu_words)
                              : nullptr;
    double *omd = om_words > 0 ? (double *)bscr->p + (3 * qn + 2 * cn + 2 * sn + 16 + 16 + flag_words + lm_words + wu_words +
                                                      f_words)
                               : nullptr;
    P.stop_level = stopd;
    P.pred_level = predd;
    P.order = orderd;
    P.lm_ctl = lmctld;
    double *o_arep = (double *)bout->p, *o_sx = o_arep + out_tot, *o_sy = o_sx + out_tot, *o_sz = o_sy + out_tot;

    int nsm = 0;
    GRPP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, st.device));
    P.status = statusd;
    P.counters = (unsigned long long *)(statusd + 16);
    P.out_tot = out_tot;
    P.outs[0] = o_arep;
    P.outs[1] = o_sx;
    P.outs[2] = o_sy;
    P.outs[3] = o_sz;
    P.n_radial = (int64_t)rad_task.size();
    P.n_mmd = (int64_t)items.size();
    P.n_entries = qtot;

    // ---------------------------------------------------------------- 2. MMD
    if (!items.empty()) {
        MmdArgs m{};
        m.items = at<MmdItem>(ib, o_items);
        m.n_items = (int)items.size();
        m.shell_L = at<int>(ib, o_shL);
        m.shell_nprim = at<int>(ib, o_shnp);
        m.shell_prim_off = at<int>(ib, o_shpo);
        m.shell_cart_off = at<int>(ib, o_shco);
        m.prim_coef = at<double>(ib, o_pc);
        m.prim_alpha = at<double>(ib, o_pa);
        m.shell_origin = at<double>(ib, o_sor);
        m.cart = at<int8_t>(ib, o_cart);
        m.pot_nprim = at<int>(ib, o_pn);
        m.pot_prim_off = at<int>(ib, o_poff);
        m.pot_powers = at<int>(ib, o_ppw);
        m.pot_coef = at<double>(ib, o_pcoef);
        m.pot_alpha = at<double>(ib, o_palpha);
        m.centre_origin = at<double>(ib, o_cor);
        m.out[0] = o_arep;
        m.out[1] = Ucd;
        m.out[2] = Scd;
        m.lmax = mmd_lmax;
        m.smax = mmd_smax;
        m.status = statusd;
        m.counters = (unsigned long long *)(statusd + 16);
        m.sched = at<uint16_t>(ib, o_msch);
        m.etab = at<int>(ib, o_met);
        m.etab_off = at<int>(ib, o_meto);
        m.rtab = at<int2>(ib, o_mrt);
        m.rtab_off = at<int>(ib, o_mrto);
        m.order = at<int>(ib, o_mord);
        m.queue = statusd + 8;
        const int wpb = 4;
        P.mmd_kpl = mmd_kpl;
        // per warp: the workspace, then 32 x KPL pair descriptors (8 bytes each)
        const size_t smem = (size_t)wpb * (mmd_ws_size(mmd_lmax, mmd_smax) + 32 * P.mmd_kpl) * sizeof(double);
        CHECK_INPUT(smem <= 200 * 1024, "type 1 workspace of this batch's angular momenta exceeds one block's shared memory");
        P.mmd = m;
        // persistent grid: the resident blocks pop items until the queue is empty
        int mmd_occ = 0;
        if (mmd_kpl == 8)
            GRPP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&mmd_occ, mmd_kernel<8, false>, 32 * wpb, smem));
        else
            GRPP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&mmd_occ, mmd_kernel<32, false>, 32 * wpb, smem));
        P.mmd_blocks = (int)std::min<int64_t>(((int64_t)items.size() + wpb - 1) / wpb, (int64_t)nsm * std::max(mmd_occ, 1));
        P.mmd_threads = 32 * wpb;
        P.mmd_smem = smem;
    }

    // ---------------------------------------------------------------- 3. outercore projections
    if (!blk_shell.empty()) {
        OcProjArgs o{};
        o.n = (int)blk_shell.size();
        o.blk_shell = at<int>(ib, o_bs);
        o.blk_ocshell = at<int>(ib, o_bo);
        o.blk_cart_off = at<int64_t>(ib, o_bco);
        o.blk_sph_off = at<int64_t>(ib, o_bso);
        o.shell_L = at<int>(ib, o_shL);
        o.shell_cart_off = at<int>(ib, o_shco);
        o.cart = at<int8_t>(ib, o_cart);
        o.S_cart = Scd;
        o.U_cart = Ucd;
        o.S_sph = Ssd;
        o.U_sph = Usd;
        P.ocp = o;
        P.ocp_blocks = (int)std::min<size_t>(blk_shell.size(), (size_t)nsm * 32);
    }

    // ---------------------------------------------------------------- 4. radial
    if (!rad_task.empty()) {
        RadialArgs r{};
        r.n_items = (int)rad_task.size();
        r.item_task = at<int>(ib, o_rt);
        r.task_a = at<int>(ib, o_ta);
        r.task_b = at<int>(ib, o_tb);
        r.task_c = at<int>(ib, o_tc);
        r.shell_L = at<int>(ib, o_shL);
        r.shell_origin = at<double>(ib, o_sor);
        r.rp_off = at<int>(ib, o_rpo);
        r.rp_n = at<int>(ib, o_rpn);
        r.rp_coef = at<double>(ib, o_rpc);
        r.rp_alpha = at<double>(ib, o_rpa);
        r.shell_nprim = at<int>(ib, o_shnp);
        r.shell_prim_off = at<int>(ib, o_shpo);
        r.prim_coef = at<double>(ib, o_pc);
        r.prim_alpha = at<double>(ib, o_pa);
        r.centre_origin = at<double>(ib, o_cor);
        r.centre_grpp = at<int>(ib, o_cg);
        r.grpp_sl_off = at<int>(ib, o_gslo);
        r.grpp_sl_n = at<int>(ib, o_gsln);
        r.sl_pot = at<int>(ib, o_slp);
        r.pot_L = at<int>(ib, o_pL);
        r.pot_nprim = at<int>(ib, o_pn);
        r.pot_prim_off = at<int>(ib, o_poff);
        r.pot_powers = at<int>(ib, o_ppw);
        r.pot_coef = at<double>(ib, o_pcoef);
        r.pot_alpha = at<double>(ib, o_palpha);
        r.q_off = at<int64_t>(ib, o_rq);
        r.n_entries = qtot;
        r.u_off = at<int64_t>(ib, o_ru);
        r.n_used = utot;
        r.ucls = at<int2>(ib, o_ucls);
        r.ulist = at<uint16_t>(ib, o_ulist);
        r.scr_units = at<ScrUnit>(ib, o_sbig);
        r.n_scr_units = (int)scr_big.size();
        r.scr_lw = scr_lw;
        r.su = at<ScrUnit>(ib, o_ssmall);
        r.su_off = at<int64_t>(ib, o_suo);
        r.n_su = (int)scr_small.size();
        r.n_su_entries = su_off.back();
        r.Q = Qd;
        r.S_prev = Spd;
        r.scr = SCd;
        r.stop_level = stopd;
        r.pred_level = nullptr;
        r.fallback_count = statusd + 4;
        r.order = nullptr;
        r.n_order = lmctld;
        r.queue = lmctld + 1;
        r.status = statusd;
        r.counters = (unsigned long long *)(statusd + 16);
        r.eflag = eflagd;
        r.walk = walkd;
        const int chunk_doubles = (rad_npot + (rad_l1 + 1) + (rad_l2 + 1) + rad_dn) * kRadRow;
        // two lists of active entries (uint16), sized for the task with most entries read
        const size_t smem = (size_t)chunk_doubles * sizeof(double) + (size_t)((4 * rad_list_max + 7) / 8) * 8;
        CHECK_INPUT(smem <= 160 * 1024, "radial grid chunk of this batch exceeds one block's shared memory");
        r.list_max = (int)rad_list_max;
        r.chunk_doubles = chunk_doubles;
        r.wu = wud;
        r.wu_npot = wu_npot;
        r.ftab = ftd;
        r.fp_off = at<int64_t>(ib, o_fpo);
        r.fp_shell = at<int>(ib, o_fps);
        r.fp_centre = at<int>(ib, o_fpc);
        r.fp_lmax = at<int>(ib, o_fpl);
        r.item_fa = at<int>(ib, o_ifa);
        r.item_fb = at<int>(ib, o_ifb);
        r.n_fpairs = (int)fp_shell.size();
        P.ftab = ftd;
        {
            int fl = 0;
            for (int v : fp_lmax) fl = std::max(fl, v);
            P.ft_smem = (size_t)(fl + 1) * kRadRow * sizeof(double);
            const int64_t nblk = (int64_t)fp_shell.size() * ((kRadGridPts + kRadThreads - 1) / kRadThreads);
            P.ft_blocks = (int)std::min<int64_t>(nblk, (int64_t)nsm * 16);
        }
        P.wu = wud;
        P.wu_grpps = ng;
        P.wu_blocks = (int)std::min<int64_t>((wu_words + 255) / 256, (int64_t)nsm * 16);
        P.rad = r;
        P.rad_blocks = (int)std::min<int64_t>((int64_t)rad_task.size(), (int64_t)nsm * 16);
        int scr_occ = 0;
        GRPP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&scr_occ, radial_screen_flat_kernel, kRadThreads, 0));
        P.scr_blocks = (int)std::min<int64_t>((su_off.back() + kRadThreads - 1) / kRadThreads, (int64_t)nsm * std::max(scr_occ, 1));
        P.scru_smem = (size_t)2 * kScrChunk * scr_lw * sizeof(double);
        int scru_occ = 0;
        GRPP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&scru_occ, radial_screen_unit_kernel, kScrUnitThreads, P.scru_smem));
        P.scru_blocks = (int)std::min<int64_t>((int64_t)scr_big.size(), (int64_t)nsm * std::max(scru_occ, 1));
        P.rad_smem = smem;
    }

    // ---------------------------------------------------------------- 5. final assembly
    {
        FinalArgs f{};
        f.n_tasks = (int)nt;
        f.task_a = at<int>(ib, o_ta);
        f.task_b = at<int>(ib, o_tb);
        f.task_c = at<int>(ib, o_tc);
        f.task_out_off = at<int64_t>(ib, o_too);
        f.task_has_ul = at<uint8_t>(ib, o_thul);
        f.task_q_off = at<int64_t>(ib, o_tqo);
        f.task_proj_a = at<int>(ib, o_tpa);
        f.task_proj_b = at<int>(ib, o_tpb);
        f.shell_L = at<int>(ib, o_shL);
        f.shell_cart_off = at<int>(ib, o_shco);
        f.shell_prim_off = at<int>(ib, o_shpo);
        f.prim_alpha = at<double>(ib, o_pa);
        f.shell_origin = at<double>(ib, o_sor);
        f.cart = at<int8_t>(ib, o_cart);
        f.centre_origin = at<double>(ib, o_cor);
        f.centre_grpp = at<int>(ib, o_cg);
        f.grpp_sl_off = at<int>(ib, o_gslo);
        f.grpp_sl_n = at<int>(ib, o_gsln);
        f.grpp_n_arep = at<int>(ib, o_gnar);
        f.sl_pot = at<int>(ib, o_slp);
        f.grpp_oc_off = at<int>(ib, o_goco);
        f.grpp_n_oc = at<int>(ib, o_gnoc);
        f.oc_L = at<int>(ib, o_ocL);
        f.oc_J = at<int>(ib, o_ocJ);
        f.oc_delta = at<double>(ib, o_del);
        f.grpp_delta_off = at<int>(ib, o_gdo);
        f.pot_L = at<int>(ib, o_pL);
        f.Q = Qd;
        f.atab_off = (const int64_t *)st.atab_off_dev.p;
        f.atab = (const double *)st.atab.p;
        f.proj_off = at<int64_t>(ib, o_poffp);
        f.S_sph = Ssd;
        f.U_sph = Usd;
        f.raw_so = opt.raw_so;
        f.arep = o_arep;
        f.so_x = o_sx;
        f.so_y = o_sy;
        f.so_z = o_sz;
        f.status = statusd;
        f.order = at<int>(ib, o_ford);
        f.queue = statusd + 9;
        f.omtab = omd;
        f.om_off = at<int64_t>(ib, o_omo);
        f.task_fpa = at<int>(ib, o_tfa);
        f.task_fpb = at<int>(ib, o_tfb);
        FinalSmem fs{};  // batch-wide layout of the omega-table kernel: RSH rows up to the largest lambda
        fs.rsh_stride = 2 * fin_lam + 1;
        fs.n_rsh = (fin_lam + 1) * fs.rsh_stride;
        P.fin = f;
        P.fin_smem_layout = fs;
        P.omtab = omd;
        P.om_pairs = (int)fp_shell.size();
        P.om_shell = at<int>(ib, o_fps);
        P.om_centre = at<int>(ib, o_fpc);
        P.om_smem = (size_t)fs.n_rsh * sizeof(double);
        P.om_blocks = (int)std::min<int64_t>((int64_t)fp_shell.size(), (int64_t)nsm * 8);
        // persistent grid per assembly group over its part of the task queue
        for (auto &G : fin_groups) {
            int occ = 0;
            GRPP_CUDA(ang_final_occupancy(G.nt, G.smem, &occ));
            G.blocks = (int)std::min<int64_t>(G.count, (int64_t)nsm * std::max(occ, 1));
        }
        // queue counters of the groups: status words 48..63 (zeroed with the status area before
        // every execution); one group per class (autotuning) takes its tasks round-robin instead
        CHECK_INPUT(opt.fin_by_class || fin_groups.size() <= 16, "more than 16 assembly launch groups");
        P.fin_queue = opt.fin_by_class ? nullptr : statusd + 48;
        P.fin_groups = fin_groups;
        P.time_groups = opt.fin_by_class != 0;
        if (P.time_groups) {
            auto &gv = st.gev[set];
            while (gv.size() < fin_groups.size() + 1) {
                cudaEvent_t e;
                GRPP_CUDA(cudaEventCreate(&e));
                gv.push_back(e);
            }
        }
    }
    return 0;
}

// Enqueue one execution of a plan on the state's stream (no host synchronisation).
int plan_launch(Plan &P)
{
    DeviceState &st = *P.st;
    cudaStream_t s = st.stream;
    cudaEvent_t *ev = st.ev[P.set];
    if (P.n_tasks == 0) return 0;
    GRPP_CUDA(cudaMemsetAsync(P.status, 0, 64 * sizeof(int), s));  // status, counters, assembly queues
    GRPP_CUDA(cudaEventRecord(ev[0], s));
    if (P.mmd_blocks > 0) {
        if (P.count_ops) {
            if (P.mmd_kpl == 8) mmd_kernel<8, true><<<P.mmd_blocks, P.mmd_threads, P.mmd_smem, s>>>(P.mmd);
            else mmd_kernel<32, true><<<P.mmd_blocks, P.mmd_threads, P.mmd_smem, s>>>(P.mmd);
        } else {
            if (P.mmd_kpl == 8) mmd_kernel<8, false><<<P.mmd_blocks, P.mmd_threads, P.mmd_smem, s>>>(P.mmd);
            else mmd_kernel<32, false><<<P.mmd_blocks, P.mmd_threads, P.mmd_smem, s>>>(P.mmd);
        }
        GRPP_CUDA(cudaGetLastError());
    }
    GRPP_CUDA(cudaEventRecord(ev[1], s));
    if (P.ocp_blocks > 0) {
        GRPP_CUDA(ang_launch_oc_proj(P.ocp_blocks, 64, s, &P.ocp, sizeof(P.ocp)));
    }
    if (P.rad_blocks > 0) {
        GRPP_CUDA(cudaMemsetAsync(P.rad.walk, 0, (size_t)P.n_radial, s));
        GRPP_CUDA(cudaMemsetAsync(P.rad.eflag, 0, (size_t)P.n_entries, s));  // unread entries stay inactive
        if (P.scru_blocks > 0) {
            radial_screen_unit_kernel<<<P.scru_blocks, kScrUnitThreads, P.scru_smem, s>>>(P.rad);
            GRPP_CUDA(cudaGetLastError());
        }
        if (P.scr_blocks > 0) {
            radial_screen_flat_kernel<<<P.scr_blocks, kRadThreads, 0, s>>>(P.rad);
            GRPP_CUDA(cudaGetLastError());
        }
        GRPP_CUDA(cudaEventRecord(ev[4], s));
        RadialArgs ra = P.rad;
        if (P.opt.radial_mode == LIBGRPP_B200_RADIAL_LEARNED) {
            if (!st.lm_ready) {
                set_error(LIBGRPP_B200_ERR_INVALID, "learned radial mode needs a level model (libgrpp_b200_set_level_model)");
                return LIBGRPP_B200_ERR_INVALID;
            }
            // predict every walked task's level, order deepest first, walk from the queue
            GRPP_CUDA(cudaMemsetAsync(P.lm_ctl, 0, 16 * sizeof(int), s));
            LevelModelDev lm{st.lm_norm, st.lm_w};
            const int pblocks = (int)std::min<int64_t>((P.n_radial + 3) / 4, (int64_t)st.nsm * 16);
            level_predict_kernel<<<pblocks, 128, 0, s>>>(P.rad, lm, P.pred_level);
            GRPP_CUDA(cudaGetLastError());
            level_order_kernel<<<1, 256, 0, s>>>((int)P.n_radial, P.pred_level, P.order, P.lm_ctl, P.lm_ctl + 2);
            GRPP_CUDA(cudaGetLastError());
            ra.order = P.order;
            ra.pred_level = P.pred_level;
            GRPP_CUDA(cudaEventRecord(ev[5], s));
        }
        if (P.wu) {
            GRPP_CUDA(nofma_launch_wu_table(P.wu_blocks, 256, s, &P.rad, sizeof(P.rad), P.wu_grpps, P.wu));
        }
        if (P.ftab) {
            GRPP_CUDA(nofma_launch_ftab(P.ft_blocks, kRadThreads, P.ft_smem, s, &P.rad, sizeof(P.rad), P.ftab));
        }
        radial_walk_kernel<<<P.rad_blocks, kRadThreads, P.rad_smem, s>>>(ra);
        GRPP_CUDA(cudaGetLastError());
    }
    GRPP_CUDA(cudaEventRecord(ev[2], s));
    if (P.omtab) {
        GRPP_CUDA(ang_launch_omega_tab(P.om_blocks, kFinThreads, P.om_smem, s, &P.fin, sizeof(P.fin), &P.fin_smem_layout,
                                       sizeof(P.fin_smem_layout), P.om_shell, P.om_centre, P.om_pairs, P.omtab));
    }
    for (size_t gi = 0; gi < P.fin_groups.size(); gi++) {
        const FinGroup &G = P.fin_groups[gi];
        FinalArgs f = P.fin;
        f.order = P.fin.order + G.first;
        f.n_tasks = G.count;
        f.queue = P.fin_queue ? P.fin_queue + gi : nullptr;
        if (P.time_groups) GRPP_CUDA(cudaEventRecord(st.gev[P.set][gi], s));
        GRPP_CUDA(ang_launch_final(G.nt, G.blocks, G.smem, s, &f, sizeof(f), &G.fs, sizeof(G.fs)));
    }
    if (P.time_groups) GRPP_CUDA(cudaEventRecord(st.gev[P.set][P.fin_groups.size()], s));
    GRPP_CUDA(cudaEventRecord(ev[3], s));
    int *hs = st.hstat[P.set];
    GRPP_CUDA(cudaMemcpyAsync(hs, P.status, 16 * sizeof(int), cudaMemcpyDeviceToHost, s));
    GRPP_CUDA(cudaMemcpyAsync(hs + 16, P.counters, kRadCntNum * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    GRPP_CUDA(cudaEventRecord(st.done[P.set], s));
    return 0;
}

// Wait for a launched execution; its timings, counters and status.
int plan_finish(Plan &P)
{
    DeviceState &st = *P.st;
    cudaEvent_t *ev = st.ev[P.set];
    if (P.n_tasks == 0) return 0;
    GRPP_CUDA(cudaEventSynchronize(st.done[P.set]));
    const int *hstatus = st.hstat[P.set];
    memcpy(P.stats.radial_counters, hstatus + 16, kRadCntNum * sizeof(unsigned long long));
    cudaEventElapsedTime(&P.stats.ms_mmd, ev[0], ev[1]);
    cudaEventElapsedTime(&P.stats.ms_radial, ev[1], ev[2]);
    if (P.rad_blocks > 0) cudaEventElapsedTime(&P.stats.ms_screen, ev[1], ev[4]);
    P.stats.ms_predict = 0.f;
    if (P.rad_blocks > 0 && P.opt.radial_mode == LIBGRPP_B200_RADIAL_LEARNED)
        cudaEventElapsedTime(&P.stats.ms_predict, ev[4], ev[5]);
    P.stats.fallbacks = hstatus[4];
    cudaEventElapsedTime(&P.stats.ms_final, ev[2], ev[3]);
    cudaEventElapsedTime(&P.stats.ms_total, ev[0], ev[3]);
    if (P.time_groups)
        for (size_t gi = 0; gi < P.fin_groups.size(); gi++)
            cudaEventElapsedTime(&P.fin_groups[gi].ms, st.gev[P.set][gi], st.gev[P.set][gi + 1]);
    P.stats.n_tasks = P.n_tasks;
    P.stats.n_radial = P.n_radial;
    P.stats.n_mmd = P.n_mmd;
    P.stats.n_entries = P.n_entries;
    if (hstatus[0] != 0) {
        set_error(LIBGRPP_B200_ERR_INVALID, "a kernel reported an index beyond its table limits");
        return LIBGRPP_B200_ERR_INVALID;
    }
    return 0;
}

int plan_execute(Plan &P)
{
    int rc = plan_launch(P);
    if (rc == 0) rc = plan_finish(P);
    return rc;
}

int plan_download(Plan &P, double *h_arep, double *h_sx, double *h_sy, double *h_sz)
{
    if (P.n_tasks == 0) return 0;
    cudaStream_t s = P.st->stream;
    double *h[4] = {h_arep, h_sx, h_sy, h_sz};
    for (int k = 0; k < 4; k++)
        if (h[k]) GRPP_CUDA(cudaMemcpyAsync(h[k], P.outs[k], P.out_tot * sizeof(double), cudaMemcpyDeviceToHost, s));
    GRPP_CUDA(cudaStreamSynchronize(s));
    return 0;
}

// Large batches run as consecutive chunks of tasks whose radial tables together stay
// below kChunkEntries entries (24 bytes of device scratch each) and kChunkTasks tasks;
// outputs land at each chunk's offset in the caller's arrays. Chunks of 32768 tasks keep
// every kernel's grid several waves deep while the host work of one chunk hides behind
// the GPU work of the previous one.
constexpr int64_t kChunkEntries = int64_t(1) << 27, kChunkTasks = int64_t(1) << 15;

int run_full_batch(const libgrpp_b200_batch_t *b, const RunOptions &opt, double *h_arep, double *h_sx, double *h_sy,
                   double *h_sz, RunStats *stats)
{
    set_error(0, "");
    int rc = 0;
    DeviceState *stp = get_state(rc);
    if (!stp) return rc;
    std::lock_guard<std::mutex> lk(stp->mu);
    for (int64_t t = 0; t < b->n_tasks; t++)
        CHECK_INPUT(b->task_a[t] >= 0 && b->task_a[t] < b->n_shells && b->task_b[t] >= 0 && b->task_b[t] < b->n_shells &&
                        b->task_c[t] >= 0 && b->task_c[t] < b->n_centres,
                    "task index out of range");
    for (int c = 0; c < b->n_centres; c++) CHECK_INPUT(b->centre_grpp[c] >= 0 && b->centre_grpp[c] < b->n_grpps, "centre GRPP index out of range");
    for (int g = 0; g < b->n_grpps; g++) {
        CHECK_INPUT(b->grpp_n_arep[g] >= 0 && b->grpp_n_so[g] >= 0, "negative potential count in a GRPP");
        for (int q = 0; q < b->grpp_n_arep[g]; q++) {
            const int pot = b->grpp_pot_list[b->grpp_arep_off[g] + q];
            CHECK_INPUT(pot >= 0 && pot < b->n_pots, "GRPP potential index out of range");
        }
        for (int q = 0; q < b->grpp_n_so[g]; q++) {
            const int pot = b->grpp_pot_list[b->grpp_so_off[g] + q];
            CHECK_INPUT(pot >= 0 && pot < b->n_pots, "GRPP potential index out of range");
        }
    }
    // chunk boundaries; a task's radial entries: sum over the centre's semilocal potentials
    // of (L+la+1)(L+lb+1)(la+lb+1)
    std::vector<std::pair<int64_t, int64_t>> chunks;
    for (int64_t t0 = 0; t0 < b->n_tasks;) {
        int64_t t1 = t0, ent = 0;
        while (t1 < b->n_tasks && t1 - t0 < kChunkTasks) {
            const int la = b->shell_L[b->task_a[t1]], lb = b->shell_L[b->task_b[t1]], g = b->centre_grpp[b->task_c[t1]];
            int64_t e = 0;
            for (int q = 0; q < b->grpp_n_arep[g] + b->grpp_n_so[g]; q++) {
                const int pot = q < b->grpp_n_arep[g] ? b->grpp_pot_list[b->grpp_arep_off[g] + q]
                                                      : b->grpp_pot_list[b->grpp_so_off[g] + q - b->grpp_n_arep[g]];
                const int L = b->pot_L[pot];
                e += (int64_t)(L + la + 1) * (L + lb + 1) * (la + lb + 1);
            }
            if (t1 > t0 && ent + e > kChunkEntries) break;
            ent += e;
            t1++;
        }
        chunks.push_back({t0, t1});
        t0 = t1;
    }
    if (chunks.empty()) chunks.push_back({0, 0});
    // chunk c uses buffer set c % 2: while the GPU runs chunk c, the host downloads chunk
    // c-1 (on the copy stream) and then prepares chunk c+1
    RunStats total;
    Plan P[2];
    int64_t out_at[2] = {0, 0}, out0 = 0;
    auto finish_and_download = [&](Plan &Q, int64_t at) -> int {
        int r = plan_finish(Q);
        if (r) return r;
        if (Q.n_tasks > 0) {
            double *h[4] = {h_arep, h_sx, h_sy, h_sz};
            GRPP_CUDA(cudaStreamWaitEvent(stp->copy_stream, stp->done[Q.set], 0));
            for (int k = 0; k < 4; k++)
                if (h[k])
                    GRPP_CUDA(cudaMemcpyAsync(h[k] + at, Q.outs[k], Q.out_tot * sizeof(double), cudaMemcpyDeviceToHost,
                                              stp->copy_stream));
            GRPP_CUDA(cudaStreamSynchronize(stp->copy_stream));
        }
        total.n_tasks += Q.stats.n_tasks;
        total.ms_total += Q.stats.ms_total;
        return 0;
    };
    for (size_t c = 0; c < chunks.size(); c++) {
        const int k = (int)(c & 1);
        libgrpp_b200_batch_t v = *b;
        v.n_tasks = chunks[c].second - chunks[c].first;
        v.task_a = b->task_a + chunks[c].first;
        v.task_b = b->task_b + chunks[c].first;
        v.task_c = b->task_c + chunks[c].first;
        P[k] = Plan();
        rc = plan_build(*stp, &v, opt, false, P[k], k);
        if (rc) return rc;
        rc = plan_launch(P[k]);
        if (rc) return rc;
        out_at[k] = out0;
        out0 += P[k].out_tot;
        if (c >= 1) {
            rc = finish_and_download(P[1 - k], out_at[1 - k]);
            if (rc) return rc;
        }
    }
    rc = finish_and_download(P[(chunks.size() - 1) & 1], out_at[(chunks.size() - 1) & 1]);
    if (stats) *stats = total;
    return rc;
}

Plan *plan_create(const libgrpp_b200_batch_t *b, const RunOptions &opt)
{
    set_error(0, "");
    int rc = 0;
    DeviceState *stp = get_state(rc);
    if (!stp) return nullptr;
    std::lock_guard<std::mutex> lk(stp->mu);
    Plan *P = new Plan();
    rc = plan_build(*stp, b, opt, true, *P);
    if (rc == 0) rc = cudaStreamSynchronize(stp->stream) == cudaSuccess ? 0 : LIBGRPP_B200_ERR_CUDA;
    if (rc) {
        plan_destroy(P);
        return nullptr;
    }
    return P;
}

void plan_set_counting(Plan *P, bool on) { P->count_ops = on; }

int plan_run(Plan *P)
{
    set_error(0, "");
    std::lock_guard<std::mutex> lk(P->st->mu);
    return plan_execute(*P);
}

int plan_outputs(Plan *P, double *h_arep, double *h_sx, double *h_sy, double *h_sz)
{
    std::lock_guard<std::mutex> lk(P->st->mu);
    return plan_download(*P, h_arep, h_sx, h_sy, h_sz);
}

// FP64 FMA throughput: 8 independent chains per thread keep the pipes busy; the
// measured rate is the denominator of the engine's FP64 roofline.
__global__ void fp64_peak_kernel(double *out, int iters, double a, double b)
{
    double x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = threadIdx.x * 1e-9 + k;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = fma(x[k], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == 12345.678) out[0] = s;  // keeps the chains live; never true for these inputs
}

int measure_fp64_peak(double *tflops)
{
    int rc = 0;
    DeviceState *stp = get_state(rc);
    if (!stp) return rc;
    std::lock_guard<std::mutex> lk(stp->mu);
    cudaStream_t s = stp->stream;
    int nsm = 0;
    GRPP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, stp->device));
    double *d = nullptr;
    GRPP_CUDA(cudaMalloc(&d, sizeof(double)));
    const int threads = 256, blocks = nsm * 8, iters = 4096;
    fp64_peak_kernel<<<blocks, threads, 0, s>>>(d, 64, 0.999999, 1e-7);
    GRPP_CUDA(cudaEventRecord(stp->ev[0][4], s));
    fp64_peak_kernel<<<blocks, threads, 0, s>>>(d, iters, 0.999999, 1e-7);
    GRPP_CUDA(cudaEventRecord(stp->ev[0][5], s));
    GRPP_CUDA(cudaEventSynchronize(stp->ev[0][5]));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, stp->ev[0][4], stp->ev[0][5]);
    cudaFree(d);
    *tflops = 2.0 * 8.0 * iters * (double)threads * blocks / (ms * 1e-3) / 1e12;
    return 0;
}

// ------------------------------------------------------------------ learned grid-level model
namespace {

// device copy of a full parameter vector: FP32 normalisation + BF16 weights
int upload_model(const float *params, float **norm, __nv_bfloat16 **w, cudaStream_t s)
{
    float *tmp = nullptr;
    GRPP_CUDA(cudaMalloc(&tmp, kLmParams * sizeof(float)));
    GRPP_CUDA(cudaMemcpyAsync(tmp, params, kLmParams * sizeof(float), cudaMemcpyHostToDevice, s));
    if (!*norm) GRPP_CUDA(cudaMalloc(norm, 2 * kLmFeat * sizeof(float)));
    if (!*w) GRPP_CUDA(cudaMalloc(w, kLmParams * sizeof(__nv_bfloat16)));
    GRPP_CUDA(cudaMemcpyAsync(*norm, tmp, 2 * kLmFeat * sizeof(float), cudaMemcpyDeviceToDevice, s));
    mlp_to_bf16_kernel<<<40, 256, 0, s>>>(tmp, *w, kLmParams);
    GRPP_CUDA(cudaGetLastError());
    GRPP_CUDA(cudaStreamSynchronize(s));
    cudaFree(tmp);
    return 0;
}

int check_model_norm(const float *params)
{
    for (int k = 0; k < kLmFeat; k++)
        if (!(params[kLmOffStd + k] > 0.f) || !std::isfinite(params[kLmOffMean + k])) {
            set_error(LIBGRPP_B200_ERR_INVALID, "level model: feature scales must be positive and means finite");
            return LIBGRPP_B200_ERR_INVALID;
        }
    return 0;
}

}  // namespace

int set_level_model(const float *params)
{
    set_error(0, "");
    int rc = 0;
    DeviceState *stp = get_state(rc);
    if (!stp) return rc;
    if ((rc = check_model_norm(params))) return rc;
    std::lock_guard<std::mutex> lk(stp->mu);
    rc = upload_model(params, &stp->lm_norm, &stp->lm_w, stp->stream);
    if (rc == 0) stp->lm_ready = true;
    return rc;
}

// Plain walk of a batch; per radial item its 12 features and the level libgrpp's
// adaptive quadrature stopped at (-1 for items whose entries all left at screening).
int level_samples(const libgrpp_b200_batch_t *b, float *features, int8_t *levels, int64_t *n_items)
{
    set_error(0, "");
    int rc = 0;
    DeviceState *stp = get_state(rc);
    if (!stp) return rc;
    std::lock_guard<std::mutex> lk(stp->mu);
    RunOptions opt;
    Plan P;
    rc = plan_build(*stp, b, opt, false, P);
    if (rc) return rc;
    *n_items = P.n_radial;
    if (P.n_radial == 0) return 0;
    GRPP_CUDA(cudaMemsetAsync(P.stop_level, -1, (size_t)P.n_radial, stp->stream));
    rc = plan_execute(P);
    if (rc) return rc;
    float *fd = nullptr;
    GRPP_CUDA(cudaMalloc(&fd, (size_t)P.n_radial * kLmFeat * sizeof(float)));
    level_features_kernel<<<(int)std::min<int64_t>((P.n_radial + 127) / 128, 4096), 128, 0, stp->stream>>>(P.rad, fd);
    GRPP_CUDA(cudaGetLastError());
    GRPP_CUDA(cudaMemcpyAsync(features, fd, (size_t)P.n_radial * kLmFeat * sizeof(float), cudaMemcpyDeviceToHost, stp->stream));
    GRPP_CUDA(cudaMemcpyAsync(levels, P.stop_level, (size_t)P.n_radial, cudaMemcpyDeviceToHost, stp->stream));
    GRPP_CUDA(cudaStreamSynchronize(stp->stream));
    cudaFree(fd);
    // items the walk skipped keep -1 (their stop level was never written)
    std::vector<uint8_t> walk((size_t)P.n_radial);
    GRPP_CUDA(cudaMemcpy(walk.data(), P.rad.walk, (size_t)P.n_radial, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < P.n_radial; i++)
        if (!walk[i]) levels[i] = -1;
    return 0;
}

namespace {

struct MlpDevice {
    float *X = nullptr, *norm = nullptr, *w = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr, *loss = nullptr;
    __nv_bfloat16 *wb = nullptr;
    int8_t *y = nullptr;
    int *idx = nullptr;
    ~MlpDevice()
    {
        for (void *p : {(void *)X, (void *)norm, (void *)w, (void *)grad, (void *)m, (void *)v, (void *)loss, (void *)wb,
                        (void *)y, (void *)idx})
            if (p) cudaFree(p);
    }
};

int mlp_setup(MlpDevice &d, const float *params, const float *X, const int8_t *y, int64_t n, cudaStream_t s)
{
    GRPP_CUDA(cudaMalloc(&d.X, (size_t)std::max<int64_t>(n, 1) * kLmFeat * sizeof(float)));
    GRPP_CUDA(cudaMalloc(&d.y, (size_t)std::max<int64_t>(n, 1)));
    GRPP_CUDA(cudaMalloc(&d.idx, (size_t)std::max<int64_t>(n, 1) * sizeof(int)));
    GRPP_CUDA(cudaMalloc(&d.norm, 2 * kLmFeat * sizeof(float)));
    GRPP_CUDA(cudaMalloc(&d.w, kLmParams * sizeof(float)));
    GRPP_CUDA(cudaMalloc(&d.wb, kLmParams * sizeof(__nv_bfloat16)));
    GRPP_CUDA(cudaMalloc(&d.grad, kLmParams * sizeof(float)));
    GRPP_CUDA(cudaMalloc(&d.m, kLmParams * sizeof(float)));
    GRPP_CUDA(cudaMalloc(&d.v, kLmParams * sizeof(float)));
    GRPP_CUDA(cudaMalloc(&d.loss, 1024 * sizeof(float)));
    if (n > 0) {
        GRPP_CUDA(cudaMemcpyAsync(d.X, X, (size_t)n * kLmFeat * sizeof(float), cudaMemcpyHostToDevice, s));
        if (y) GRPP_CUDA(cudaMemcpyAsync(d.y, y, (size_t)n, cudaMemcpyHostToDevice, s));
    }
    GRPP_CUDA(cudaMemcpyAsync(d.norm, params, 2 * kLmFeat * sizeof(float), cudaMemcpyHostToDevice, s));
    GRPP_CUDA(cudaMemcpyAsync(d.w, params, kLmParams * sizeof(float), cudaMemcpyHostToDevice, s));
    mlp_to_bf16_kernel<<<40, 256, 0, s>>>(d.w, d.wb, kLmParams);
    GRPP_CUDA(cudaGetLastError());
    GRPP_CUDA(cudaMemsetAsync(d.grad, 0, kLmParams * sizeof(float), s));
    GRPP_CUDA(cudaMemsetAsync(d.m, 0, kLmParams * sizeof(float), s));
    GRPP_CUDA(cudaMemsetAsync(d.v, 0, kLmParams * sizeof(float), s));
    GRPP_CUDA(cudaMemsetAsync(d.loss, 0, 1024 * sizeof(float), s));
    return 0;
}

int check_labels(const int8_t *y, int64_t n)
{
    for (int64_t i = 0; i < n; i++)
        if (y[i] < 0 || y[i] >= kLmOut) {
            set_error(LIBGRPP_B200_ERR_INVALID, "level labels must be 0..8");
            return LIBGRPP_B200_ERR_INVALID;
        }
    return 0;
}

}  // namespace

// Gradient (w.r.t. the BF16-rounded weights) and mean cross-entropy of the model on n samples.
int mlp_grad(const float *params, const float *X, const int8_t *y, int n, float *grad, float *loss)
{
    set_error(0, "");
    int rc = 0;
    DeviceState *stp = get_state(rc);
    if (!stp) return rc;
    if (n <= 0) {
        set_error(LIBGRPP_B200_ERR_INVALID, "mlp_grad needs at least one sample");
        return LIBGRPP_B200_ERR_INVALID;
    }
    if ((rc = check_model_norm(params)) || (rc = check_labels(y, n))) return rc;
    std::lock_guard<std::mutex> lk(stp->mu);
    cudaStream_t s = stp->stream;
    MlpDevice d;
    if ((rc = mlp_setup(d, params, X, y, n, s))) return rc;
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    GRPP_CUDA(cudaMemcpyAsync(d.idx, idx.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
    MlpTrainArgs t{d.X, d.y, d.idx, n, 0, n, d.norm, d.wb, d.grad, d.loss};
    mlp_train_kernel<<<(n + kLmTrainSamples - 1) / kLmTrainSamples, kLmTrainThreads, mlp_train_smem_bytes(), s>>>(t);
    GRPP_CUDA(cudaGetLastError());
    GRPP_CUDA(cudaMemcpyAsync(grad, d.grad, kLmParams * sizeof(float), cudaMemcpyDeviceToHost, s));
    GRPP_CUDA(cudaMemcpyAsync(loss, d.loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    GRPP_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < kLmOffW1; i++) grad[i] = 0.f;
    return 0;
}

// Adam training of the model on n (features, level) pairs; params in: initial weights and
// the feature normalisation, out: trained FP32 master weights. epoch_loss[e] = mean
// cross-entropy seen during epoch e. Minibatches of `batch` samples, reshuffled per epoch.
int mlp_train(const float *X, const int8_t *y, int64_t n, int epochs, int batch, float lr, uint32_t seed,
              float *params, float *epoch_loss)
{
    set_error(0, "");
    int rc = 0;
    DeviceState *stp = get_state(rc);
    if (!stp) return rc;
    if (n <= 0 || epochs <= 0 || epochs > 1024 || batch <= 0 || n > (int64_t)INT32_MAX) {
        set_error(LIBGRPP_B200_ERR_INVALID, "mlp_train: need n in 1..2^31-1, epochs in 1..1024, batch > 0");
        return LIBGRPP_B200_ERR_INVALID;
    }
    if ((rc = check_model_norm(params)) || (rc = check_labels(y, n))) return rc;
    std::lock_guard<std::mutex> lk(stp->mu);
    cudaStream_t s = stp->stream;
    MlpDevice d;
    if ((rc = mlp_setup(d, params, X, y, n, s))) return rc;
    std::vector<int> idx((size_t)n);
    uint64_t state = 0x9E3779B97F4A7C15ull ^ seed;
    auto rnd = [&state]() {  // splitmix64
        state += 0x9E3779B97F4A7C15ull;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    const float b1 = 0.9f, b2 = 0.999f;
    float p1 = 1.f, p2 = 1.f;
    for (int ep = 0; ep < epochs; ep++) {
        for (int64_t i = 0; i < n; i++) idx[i] = (int)i;
        for (int64_t i = n - 1; i > 0; i--) std::swap(idx[i], idx[rnd() % (uint64_t)(i + 1)]);
        GRPP_CUDA(cudaMemcpyAsync(d.idx, idx.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s));
        int steps = 0;
        for (int64_t b0 = 0; b0 < n; b0 += batch) {
            const int bsz = (int)std::min<int64_t>(batch, n - b0);
            MlpTrainArgs t{d.X, d.y, d.idx, (int)n, (int)b0, bsz, d.norm, d.wb, d.grad, d.loss + ep};
            mlp_train_kernel<<<(bsz + kLmTrainSamples - 1) / kLmTrainSamples, kLmTrainThreads, mlp_train_smem_bytes(), s>>>(t);
            GRPP_CUDA(cudaGetLastError());
            p1 *= b1;
            p2 *= b2;
            AdamArgs ad{d.w, d.wb, d.grad, d.m, d.v, lr, b1, b2, 1e-8f, 1.f - p1, 1.f - p2};
            mlp_adam_kernel<<<40, 256, 0, s>>>(ad);
            GRPP_CUDA(cudaGetLastError());
            steps++;
        }
        float l = 0.f;
        GRPP_CUDA(cudaMemcpyAsync(&l, d.loss + ep, sizeof(float), cudaMemcpyDeviceToHost, s));
        GRPP_CUDA(cudaStreamSynchronize(s));
        if (epoch_loss) epoch_loss[ep] = l / (float)steps;
    }
    GRPP_CUDA(cudaMemcpyAsync(params + kLmOffW1, d.w + kLmOffW1, kLmNet * sizeof(float), cudaMemcpyDeviceToHost, s));
    GRPP_CUDA(cudaStreamSynchronize(s));
    return 0;
}

namespace {
__global__ void mlp_predict_kernel(LevelModelDev m, const float *X, int n, int8_t *pred)
{
    __shared__ float hbuf[4][2 * kLmHid];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = blockIdx.x * 4 + warp; i < n; i += gridDim.x * 4) {
        const int l = mlp_forward_warp(m, X + (size_t)i * kLmFeat, hbuf[warp], lane);
        if (lane == 0) pred[i] = (int8_t)l;
        __syncwarp();
    }
}
}  // namespace

// Predicted level (argmax) of n feature rows, with the BF16 inference path of the walk.
int mlp_predict(const float *params, const float *X, int64_t n, int8_t *pred)
{
    set_error(0, "");
    int rc = 0;
    DeviceState *stp = get_state(rc);
    if (!stp) return rc;
    if (n <= 0 || n > (int64_t)INT32_MAX) {
        set_error(LIBGRPP_B200_ERR_INVALID, "mlp_predict: need n in 1..2^31-1");
        return LIBGRPP_B200_ERR_INVALID;
    }
    if ((rc = check_model_norm(params))) return rc;
    std::lock_guard<std::mutex> lk(stp->mu);
    cudaStream_t s = stp->stream;
    MlpDevice d;
    if ((rc = mlp_setup(d, params, X, nullptr, n, s))) return rc;
    int8_t *pd = nullptr;
    GRPP_CUDA(cudaMalloc(&pd, (size_t)n));
    LevelModelDev lm{d.norm, d.wb};
    mlp_predict_kernel<<<(int)std::min<int64_t>((n + 3) / 4, (int64_t)stp->nsm * 16), 128, 0, s>>>(lm, d.X, (int)n, pd);
    GRPP_CUDA(cudaGetLastError());
    GRPP_CUDA(cudaMemcpyAsync(pred, pd, (size_t)n, cudaMemcpyDeviceToHost, s));
    GRPP_CUDA(cudaStreamSynchronize(s));
    cudaFree(pd);
    return 0;
}

// Density-contracted gradient pieces of a task list whose GRPP blocks come from the
// sub-task batch `sub` (the differentiated shell pairs): out24[t] = G[side][k][m] of
// task t (gradient.cuh). cart_tab: [kMaxL+1][kGradMaxCart][3][3] component table.
int run_grad_contract(const libgrpp_b200_batch_t *sub, const RunOptions &opt, const GradTaskHost *tasks,
                      int64_t n_tasks, const int *cart_tab, const double *D, int64_t n_bf, double *out24)
{
    set_error(0, "");
    int rc = 0;
    DeviceState *stp = get_state(rc);
    if (!stp) return rc;
    std::lock_guard<std::mutex> lk(stp->mu);
    cudaStream_t s = stp->stream;
    Plan P;
    rc = plan_build(*stp, sub, opt, false, P);
    if (rc) return rc;
    rc = plan_execute(P);
    if (rc) return rc;
    if (n_tasks == 0) return 0;
    static_assert(kGradMaxL == kMaxL && kGradTabCart == kGradMaxCart, "gradient component table");
    const size_t tab_n = (size_t)(kMaxL + 1) * kGradMaxCart * 9;
    const size_t bytes = n_tasks * sizeof(GradTask) + tab_n * sizeof(int) + (size_t)n_bf * n_bf * sizeof(double) +
                         (size_t)n_tasks * 24 * sizeof(double) + 4 * 256;
    GRPP_CUDA(stp->grad.ensure(bytes));  // kept across calls: no allocation per chunk
    char *q = (char *)stp->grad.p;
    auto take = [&q](size_t n) {
        char *r = q;
        q += (n + 255) & ~(size_t)255;
        return r;
    };
    GradTask *td = (GradTask *)take(n_tasks * sizeof(GradTask));
    int *tabd = (int *)take(tab_n * sizeof(int));
    double *Dd = (double *)take((size_t)n_bf * n_bf * sizeof(double));
    double *gd = (double *)take((size_t)n_tasks * 24 * sizeof(double));
    static_assert(sizeof(GradTask) == sizeof(GradTaskHost), "GradTask layout");
    GRPP_CUDA(cudaMemcpyAsync(td, tasks, n_tasks * sizeof(GradTask), cudaMemcpyHostToDevice, s));
    GRPP_CUDA(cudaMemcpyAsync(tabd, cart_tab, tab_n * sizeof(int), cudaMemcpyHostToDevice, s));
    GRPP_CUDA(cudaMemcpyAsync(Dd, D, (size_t)n_bf * n_bf * sizeof(double), cudaMemcpyHostToDevice, s));
    GradArgs ga{};
    ga.tasks = td;
    ga.n_tasks = (int)n_tasks;
    ga.cart_tab = tabd;
    ga.sub_off = P.fin.task_out_off;
    for (int m = 0; m < 4; m++) ga.out[m] = P.outs[m];
    ga.D = Dd;
    ga.n_bf = n_bf;
    ga.g = gd;
    grad_contract_kernel<<<(int)std::min<int64_t>((n_tasks + 3) / 4, (int64_t)stp->nsm * 32), 128, 0, s>>>(ga);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out24, gd, (size_t)n_tasks * 24 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error(LIBGRPP_B200_ERR_CUDA, std::string("gradient contraction: ") + cudaGetErrorString(e));
        return LIBGRPP_B200_ERR_CUDA;
    }
    return 0;
}

// ------------------------------------------------------------------ one-electron batches
namespace {

// shells and tasks of a batch packed for the one-electron kernels (Cartesian lists as int8,
// task blocks laid out as in run_full_batch)
struct OneePack {
    std::vector<int> sL, snp, spo, sco, ta, tb, tc;
    std::vector<double> pc, pa, so;
    std::vector<int8_t> cart;
    std::vector<int64_t> off;
    int lmax_pair = 0;
};

int onee_pack(const libgrpp_b200_batch_t *b, bool need_centres, int lmax_shell, OneePack &k)
{
    const int64_t nt = b->n_tasks;
    auto bad = [](const char *m) {
        set_error(LIBGRPP_B200_ERR_INVALID, m);
        return LIBGRPP_B200_ERR_INVALID;
    };
    if (nt < 0) return bad("negative task count");
    if (nt > ((int64_t)1 << 31) - 1) return bad("more than 2^31 - 1 tasks in one call");
    if (nt == 0) return 0;
    if (b->n_shells <= 0 || (need_centres && b->n_centres <= 0)) return bad("empty batch description");
    const int ns = b->n_shells;
    k.sL.assign(b->shell_L, b->shell_L + ns);
    k.snp.assign(b->shell_nprim, b->shell_nprim + ns);
    k.spo.assign(b->shell_prim_off, b->shell_prim_off + ns);
    k.sco.resize(ns);
    k.so.assign(b->shell_origin, b->shell_origin + 3 * ns);
    int tot = 0;
    for (int i = 0; i < ns; i++) {
        if (k.sL[i] < 0 || k.sL[i] > lmax_shell) return bad("shell angular momentum outside the supported range");
        if (k.snp[i] < 0 || k.snp[i] > kRadMaxPrims || k.spo[i] < 0) return bad("shell primitive count or offset out of range");
        tot = std::max(tot, k.spo[i] + k.snp[i]);
        k.sco[i] = (int)(k.cart.size() / 3);
        for (int q = 0; q < 3 * ncart(k.sL[i]); q++) {
            const int v = b->cart_list[3 * b->shell_cart_off[i] + q];
            if (v < 0 || v > k.sL[i]) return bad("invalid Cartesian component list");
            k.cart.push_back((int8_t)v);
        }
    }
    k.pc.assign(b->prim_coef, b->prim_coef + tot);
    k.pa.assign(b->prim_alpha, b->prim_alpha + tot);
    k.ta.assign(b->task_a, b->task_a + nt);
    k.tb.assign(b->task_b, b->task_b + nt);
    k.off.assign(nt + 1, 0);
    if (need_centres) k.tc.assign(b->task_c, b->task_c + nt);
    for (int64_t t = 0; t < nt; t++) {
        if (k.ta[t] < 0 || k.ta[t] >= ns || k.tb[t] < 0 || k.tb[t] >= ns) return bad("task index out of range");
        if (need_centres && (k.tc[t] < 0 || k.tc[t] >= b->n_centres)) return bad("task centre index out of range");
        k.off[t + 1] = k.off[t] + (int64_t)ncart(k.sL[k.ta[t]]) * ncart(k.sL[k.tb[t]]);
        k.lmax_pair = std::max(k.lmax_pair, k.sL[k.ta[t]] + k.sL[k.tb[t]]);
    }
    return 0;
}

struct OneeUpload {
    char *dev = nullptr;
    std::vector<char> host;
    size_t used = 0;
    template <typename T>
    size_t add(const std::vector<T> &v)
    {
        const size_t o = (used + 255) & ~size_t(255);
        used = o + std::max<size_t>(v.size(), 1) * sizeof(T);
        host.resize(used);
        if (!v.empty()) memcpy(host.data() + o, v.data(), v.size() * sizeof(T));
        return o;
    }
    size_t reserve(size_t bytes)
    {
        const size_t o = (used + 255) & ~size_t(255);
        used = o + std::max<size_t>(bytes, 8);
        return o;
    }
    template <typename T>
    T *at(size_t o) const
    {
        return (T *)(dev + o);
    }
};

}  // namespace

int run_onee_batch(const libgrpp_b200_batch_t *b, int kind, double *h0, double *h1, double *h2)
{
    set_error(0, "");
    if (kind < kOneeOverlap || kind > kOneeMomentum) {
        set_error(LIBGRPP_B200_ERR_INVALID, "unknown one-electron integral kind");
        return LIBGRPP_B200_ERR_INVALID;
    }
    OneePack k;
    int rc = onee_pack(b, false, kMaxL, k);
    if (rc || b->n_tasks == 0) return rc;
    DeviceState *stp = get_state(rc);
    if (!stp) return rc;
    std::lock_guard<std::mutex> lk(stp->mu);
    cudaStream_t s = stp->stream;
    const int64_t nt = b->n_tasks, nout = k.off[nt];
    const int nouts = kind == kOneeMomentum ? 3 : 1;
    OneeUpload u;
    const size_t oL = u.add(k.sL), onp = u.add(k.snp), opo = u.add(k.spo), oco = u.add(k.sco), opc = u.add(k.pc),
                 opa = u.add(k.pa), oso = u.add(k.so), ocart = u.add(k.cart), ota = u.add(k.ta), otb = u.add(k.tb),
                 ooff = u.add(k.off);
    const size_t in_bytes = u.used;
    const size_t oout = u.reserve((size_t)nouts * nout * sizeof(double));
    GRPP_CUDA(stp->onee.ensure(u.used));
    u.dev = (char *)stp->onee.p;
    GRPP_CUDA(cudaMemcpyAsync(u.dev, u.host.data(), in_bytes, cudaMemcpyHostToDevice, s));
    OneeArgs a{};
    a.n_tasks = (int)nt;
    a.kind = kind;
    a.task_a = u.at<int>(ota);
    a.task_b = u.at<int>(otb);
    a.out_off = u.at<int64_t>(ooff);
    a.shell_L = u.at<int>(oL);
    a.shell_nprim = u.at<int>(onp);
    a.shell_prim_off = u.at<int>(opo);
    a.shell_cart_off = u.at<int>(oco);
    a.prim_coef = u.at<double>(opc);
    a.prim_alpha = u.at<double>(opa);
    a.shell_origin = u.at<double>(oso);
    a.cart = u.at<int8_t>(ocart);
    a.out0 = u.at<double>(oout);
    a.out1 = a.out0 + nout;
    a.out2 = a.out1 + nout;
    const int blocks = (int)std::min<int64_t>((nt + kOneeWarps - 1) / kOneeWarps, (int64_t)stp->nsm * 16);
    onee_os_kernel<<<blocks, 32 * kOneeWarps, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    double *hs[3] = {h0, h1, h2};
    for (int m = 0; m < nouts && e == cudaSuccess; m++)
        e = cudaMemcpyAsync(hs[m], a.out0 + m * nout, nout * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error(LIBGRPP_B200_ERR_CUDA, std::string("one-electron integrals: ") + cudaGetErrorString(e));
        return LIBGRPP_B200_ERR_CUDA;
    }
    return 0;
}

int run_type1_numeric_batch(const libgrpp_b200_batch_t *b, int model, const double *centre_param, double tol,
                            double pair_skip, double *h_out)
{
    set_error(0, "");
    auto bad = [](const char *m) {
        set_error(LIBGRPP_B200_ERR_INVALID, m);
        return LIBGRPP_B200_ERR_INVALID;
    };
    if (model < kPotGrpp || model > kPotFermiBubble) return bad("unknown radially local potential model");
    OneePack k;
    int rc = onee_pack(b, true, kMaxL, k);
    if (rc || b->n_tasks == 0) return rc;
    if (k.lmax_pair > kT1MaxLam) return bad("numeric type 1 integrals need L_A + L_B <= 12");
    if (model != kPotGrpp && !centre_param) return bad("nuclear model parameters missing");
    // the centres' radially local potentials: U_L of each centre's GRPP (terms with |c| > 1e-14,
    // as libgrpp_shrink_potential keeps them), or the model parameters
    const int nc = b->n_centres;
    std::vector<double> cor(b->centre_origin, b->centre_origin + 3 * nc), cpar((size_t)4 * nc, 0.0);
    std::vector<int> cpo(nc, 0), cpn(nc, 0), ppw;
    std::vector<double> pco, pal;
    for (int c = 0; c < nc; c++) {
        if (model != kPotGrpp) {
            for (int q = 0; q < 4; q++) cpar[4 * c + q] = centre_param[4 * c + q];
            continue;
        }
        const int g = b->centre_grpp[c];
        if (g < 0 || g >= b->n_grpps) return bad("centre GRPP index out of range");
        cpo[c] = (int)pco.size();
        const int p = b->grpp_UL[g];
        if (p < 0) continue;
        if (p >= b->n_pots) return bad("GRPP potential index out of range");
        for (int q = 0; q < b->pot_nprim[p]; q++) {
            const int o = b->pot_prim_off[p] + q;
            if (b->pot_powers[o] < 0 || b->pot_powers[o] > 2) return bad("potential power n must be 0, 1 or 2");
            if (std::fabs(b->pot_coef[o]) <= kZeroThresh) continue;
            ppw.push_back(b->pot_powers[o]);
            pco.push_back(b->pot_coef[o]);
            pal.push_back(b->pot_alpha[o]);
        }
        cpn[c] = (int)pco.size() - cpo[c];
    }
    DeviceState *stp = get_state(rc);
    if (!stp) return rc;
    std::lock_guard<std::mutex> lk(stp->mu);
    cudaStream_t s = stp->stream;
    const int64_t nt = b->n_tasks, nout = k.off[nt];
    const int Lt = k.lmax_pair;
    const int64_t n_ang = (int64_t)(Lt + 1) * (2 * Lt + 1) * n_abc(Lt);
    OneeUpload u;
    const size_t oL = u.add(k.sL), onp = u.add(k.snp), opo = u.add(k.spo), oco = u.add(k.sco), opc = u.add(k.pc),
                 opa = u.add(k.pa), oso = u.add(k.so), ocart = u.add(k.cart), ota = u.add(k.ta), otb = u.add(k.tb),
                 otc = u.add(k.tc), ooff = u.add(k.off), ocor = u.add(cor), ocpar = u.add(cpar), ocpo = u.add(cpo),
                 ocpn = u.add(cpn), oppw = u.add(ppw), opco = u.add(pco), opal = u.add(pal);
    const size_t in_bytes = u.used;
    const size_t oang = u.reserve(n_ang * sizeof(double)), oout = u.reserve(nout * sizeof(double));
    GRPP_CUDA(stp->onee.ensure(u.used));
    u.dev = (char *)stp->onee.p;
    GRPP_CUDA(cudaMemcpyAsync(u.dev, u.host.data(), in_bytes, cudaMemcpyHostToDevice, s));
    type1_ang_kernel<<<(int)std::min<int64_t>((n_ang + 255) / 256, 4096), 256, 0, s>>>(Lt, u.at<double>(oang));
    Type1NumArgs a{};
    a.n_tasks = (int)nt;
    a.model = model;
    a.task_a = u.at<int>(ota);
    a.task_b = u.at<int>(otb);
    a.task_c = u.at<int>(otc);
    a.out_off = u.at<int64_t>(ooff);
    a.shell_L = u.at<int>(oL);
    a.shell_nprim = u.at<int>(onp);
    a.shell_prim_off = u.at<int>(opo);
    a.shell_cart_off = u.at<int>(oco);
    a.prim_coef = u.at<double>(opc);
    a.prim_alpha = u.at<double>(opa);
    a.shell_origin = u.at<double>(oso);
    a.cart = u.at<int8_t>(ocart);
    a.centre_origin = u.at<double>(ocor);
    a.centre_param = u.at<double>(ocpar);
    a.centre_pot_off = u.at<int>(ocpo);
    a.centre_pot_n = u.at<int>(ocpn);
    a.pot_pow = u.at<int>(oppw);
    a.pot_coef = u.at<double>(opco);
    a.pot_alpha = u.at<double>(opal);
    a.fermi = stp->fermi;
    a.ang1 = u.at<double>(oang);
    a.lmax_tab = Lt;
    a.tol = tol;
    a.pair_skip = pair_skip;
    a.out = u.at<double>(oout);
    const size_t smem = (size_t)t1_smem_doubles(Lt) * sizeof(double);
    type1_num_kernel<<<(int)std::min<int64_t>(nt, (int64_t)stp->nsm * 8), kT1Threads, smem, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_out, a.out, nout * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error(LIBGRPP_B200_ERR_CUDA, std::string("numeric type 1 integrals: ") + cudaGetErrorString(e));
        return LIBGRPP_B200_ERR_CUDA;
    }
    return 0;
}

const RunStats *plan_stats(const Plan *P) { return &P->stats; }
int64_t plan_h2d_bytes(const Plan *P) { return P->h2d_bytes; }

void *host_alloc(size_t bytes)
{
    set_error(0, "");
    void *p = nullptr;
    const cudaError_t e = cudaHostAlloc(&p, std::max<size_t>(bytes, 1), cudaHostAllocDefault);
    if (e != cudaSuccess) {
        set_error(LIBGRPP_B200_ERR_CUDA, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
        return nullptr;
    }
    return p;
}

void host_free(void *p)
{
    if (p) cudaFreeHost(p);
}

int set_device(int device)
{
    GRPP_CUDA(cudaSetDevice(device));
    return 0;
}

// Assembly autotuner: every class of the batch runs with each block size as a launch of its
// own (round-robin over the class's tasks, CUDA events around each launch), twice; the second
// timing counts. The fastest block size per class goes into the device's table, which the
// planner uses for later batches. Rows: class key, tasks, ms at 128, 256, 512 threads, choice.
int autotune_assembly(const libgrpp_b200_batch_t *b, int radial_mode, std::vector<std::array<double, 6>> &rows)
{
    set_error(0, "");
    int rc = 0;
    DeviceState *stp = get_state(rc);
    if (!stp) return rc;
    std::lock_guard<std::mutex> lk(stp->mu);
    const int sizes[3] = {128, 256, 512};
    std::map<int, std::array<double, 6>> tab;
    for (int v = 0; v < 3; v++) {
        RunOptions o;
        o.radial_mode = radial_mode;
        o.fin_nt = sizes[v];
        o.fin_by_class = 1;
        Plan P;
        rc = plan_build(*stp, b, o, true, P);
        if (rc == 0) rc = plan_execute(P);
        if (rc == 0) rc = plan_execute(P);
        if (rc == 0)
            for (const FinGroup &G : P.fin_groups) {
                auto &r = tab[G.key];
                r[0] = G.key;
                r[1] = G.count;
                r[2 + v] = G.ms;
            }
        for (DevBuf *d : {&P.in, &P.scratch, &P.out})
            if (d->p) cudaFree(d->p);
        if (rc) return rc;
    }
    rows.clear();
    for (auto &kv : tab) {
        auto r = kv.second;
        int best = 0;
        for (int v = 1; v < 3; v++)
            if (r[2 + v] < r[2 + best]) best = v;
        r[5] = sizes[best];
        stp->fin_tune[kv.first] = sizes[best];
        rows.push_back(r);
    }
    return 0;
}

void autotune_reset()
{
    int rc = 0;
    DeviceState *stp = get_state(rc);
    if (!stp) return;
    std::lock_guard<std::mutex> lk(stp->mu);
    stp->fin_tune.clear();
}

void plan_destroy(Plan *P)
{
    if (!P) return;
    for (DevBuf *d : {&P->in, &P->scratch, &P->out})
        if (d->p) cudaFree(d->p);
    delete P;
}


}  // namespace grpp
