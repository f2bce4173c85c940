// Y-bus value assembly on the device and the gapk_ybus_* C ABI.
//
// One thread per (scenario, CSR slot).  An off-diagonal slot holds the stamp of the one
// branch triplet that produced it; a diagonal slot sums its bus's shunt and branch-end stamps
// sequentially in the reference's accumulation order (shunts in appliance order, then branch
// ends in branch order), so the result is deterministic and, in reference mode, bit-identical
// to src/admittance/cpu/cpu_admittance_matrix.cpp:88-145.  No atomics.
//
// All reference-mode arithmetic uses explicitly rounded intrinsics (__dmul_rn, __dadd_rn,
// __ddiv_rn) so that no multiply-add is contracted into an FMA: the reference computes
// r*r + x*x with two roundings.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "../../include/gapk.h"
#include "internal.h"

namespace gapk {
namespace {

struct Stamps {
    double2 ff, tt, ft, tf;
};

__device__ __forceinline__ Stamps branch_stamps(const double* __restrict__ br, int mode) {
    const double r = br[0], x = br[1], g = br[2], b = br[3], k = br[4], th = br[5];
    const double z2 = __dadd_rn(__dmul_rn(r, r), __dmul_rn(x, x));
    double yr = 0.0, yi = 0.0;
    if (z2 > 1e-12) {
        yr = __ddiv_rn(r, z2);
        yi = __ddiv_rn(-x, z2);
    }
    // end stamp y + g1 + j b1/2 (cpu_admittance_matrix.cpp:130-135)
    const double er = __dadd_rn(__dadd_rn(yr, g), 0.0);
    const double ei = __dadd_rn(__dadd_rn(yi, 0.0), __ddiv_rn(b, 2.0));
    Stamps s;
    if (mode == GAPK_YBUS_REFERENCE || (k == 1.0 && th == 0.0)) {
        s.ff = make_double2(er, ei);
        s.tt = s.ff;
        s.ft = make_double2(-yr, -yi);
        s.tf = s.ft;
    } else {
        // tap t = k e^{j th} on the from side: Y_ff = (y+ysh)/k^2, Y_ft = -y/conj(t),
        // Y_tf = -y/t, Y_tt = y+ysh
        double sn, cs;
        sincos(th, &sn, &cs);
        const double k2 = k * k;
        s.ff = make_double2(er / k2, ei / k2);
        s.tt = make_double2(er, ei);
        // -y / conj(t) = -y * t / k^2 ;  -y / t = -y * conj(t) / k^2
        const double tr = k * cs, ti = k * sn;
        s.ft = make_double2(-(yr * tr - yi * ti) / k2, -(yr * ti + yi * tr) / k2);
        s.tf = make_double2(-(yr * tr + yi * ti) / k2, -(yi * tr - yr * ti) / k2);
    }
    return s;
}

__global__ void k_ybus(int nnz, int n_scen, const int* __restrict__ slot_src,
                       const int* __restrict__ diag_ptr, const int* __restrict__ diag_src,
                       const double* __restrict__ br, long long br_stride,
                       const double* __restrict__ sh, long long sh_stride, int mode,
                       double scale, double2* __restrict__ out, long long out_stride) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long long)nnz * n_scen) return;
    const int s = (int)(tid / nnz), p = (int)(tid % nnz);
    const double* B = br + (size_t)s * br_stride;
    const double* S = sh + (size_t)s * sh_stride;
    const int src = slot_src[p];
    double vr, vi;
    if (src >= 0) {
        const Stamps st = branch_stamps(B + (size_t)(src >> 1) * 6, mode);
        const double2 v = (src & 1) ? st.tf : st.ft;
        vr = v.x;
        vi = v.y;
    } else {
        const int i = -src - 1;
        vr = 0.0;
        vi = 0.0;
        for (int c = diag_ptr[i]; c < diag_ptr[i + 1]; ++c) {
            const int d = diag_src[c];
            if (d < 0) {
                const double* q = S + (size_t)(-d - 1) * 2;
                vr = __dadd_rn(vr, q[0]);
                vi = __dadd_rn(vi, q[1]);
            } else {
                const Stamps st = branch_stamps(B + (size_t)(d >> 1) * 6, mode);
                const double2 v = (d & 1) ? st.tt : st.ff;
                vr = __dadd_rn(vr, v.x);
                vi = __dadd_rn(vi, v.y);
            }
        }
    }
    if (scale != 1.0) {
        vr = __dmul_rn(vr, scale);
        vi = __dmul_rn(vi, scale);
    }
    out[(size_t)s * out_stride + p] = make_double2(vr, vi);
}

// Branch status changes on existing values, one thread per (scenario, touched CSR slot).
// Each thread applies the deltas of its slot in change order, so the result of every slot is
// the one the reference's sequential loop gives (src/admittance/cpu/cpu_admittance_matrix.cpp:
// 214-297: different slots never interact), whatever the number of threads.
//   item  = (scenario, slot, first, last) into seg; seg[e] = change index << 2 | role, role
//           0 / 1 the from / to diagonal, 2 the (from, to) entry, 3 the (to, from) entry
//   prm   = (r1, x1, g1, b1, k, theta, status) per change, Ohm / S
// Delta of one change (sign + when the branch comes into service, - when it leaves):
//   GAPK_DELTA_REFERENCE   the reference's update: diagonals y + g1 + j b1 + j b1/2 (unlike its
//                          build, which stamps y + g1 + j b1/2), off-diagonals -y; taps ignored
//   GAPK_DELTA_FIXED       the builder's own stamps, taps ignored (GAPK_YBUS_REFERENCE)
//   GAPK_DELTA_FIXED_TAPS  the builder's pi-model stamps with the tap (GAPK_YBUS_TAPS)
// scale multiplies every delta (1 = Siemens, Z_base = per unit).
__device__ __forceinline__ double2 change_delta(const double* __restrict__ q, int role, int mode) {
    double2 d;
    if (mode == GAPK_DELTA_REFERENCE) {
        const double r = q[0], x = q[1], g = q[2], b = q[3];
        const double z2 = __dadd_rn(__dmul_rn(r, r), __dmul_rn(x, x));
        double yr = 0.0, yi = 0.0;
        if (z2 > 1e-12) {
            yr = __ddiv_rn(r, z2);
            yi = __ddiv_rn(-x, z2);
        }
        if (role < 2) {
            // (y + (g1 + j b1)) + j b1/2, each sum rounded as the reference's complex adds
            d = make_double2(__dadd_rn(__dadd_rn(yr, g), 0.0),
                             __dadd_rn(__dadd_rn(yi, b), __ddiv_rn(b, 2.0)));
        } else {
            d = make_double2(-yr, -yi);
        }
    } else {
        const Stamps st = branch_stamps(q, mode == GAPK_DELTA_FIXED ? GAPK_YBUS_REFERENCE
                                                                    : GAPK_YBUS_TAPS);
        d = role == 0 ? st.ff : role == 1 ? st.tt : role == 2 ? st.ft : st.tf;
    }
    if (q[6] == 0.0) d = make_double2(-d.x, -d.y);
    return d;
}

__global__ void k_ybus_delta(int n_items, const int4* __restrict__ items,
                             const int* __restrict__ seg, const double* __restrict__ prm,
                             int mode, double scale, double2* __restrict__ values,
                             long long stride) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_items) return;
    const int4 it = items[t];
    double2* v = values + (size_t)it.x * stride + it.y;
    double vr = v->x, vi = v->y;
    for (int e = it.z; e < it.w; ++e) {
        const int c = seg[e] >> 2, role = seg[e] & 3;
        double2 d = change_delta(prm + (size_t)c * 7, role, mode);
        if (scale != 1.0) d = make_double2(__dmul_rn(d.x, scale), __dmul_rn(d.y, scale));
        if (mode == GAPK_DELTA_REFERENCE && role >= 2) {
            // values[idx] -= series change: -(+-y)
            vr = __dsub_rn(vr, -d.x);
            vi = __dsub_rn(vi, -d.y);
        } else {
            vr = __dadd_rn(vr, d.x);
            vi = __dadd_rn(vi, d.y);
        }
    }
    *v = make_double2(vr, vi);
}

}  // namespace
}  // namespace gapk

using namespace gapk;

struct gapk_ybus_s {
    YbusPatternHost h;
    int device = -1;
    void* d_slot_src = nullptr;
    void* d_diag_ptr = nullptr;
    void* d_diag_src = nullptr;
    ~gapk_ybus_s() {
        if (d_slot_src) cudaFree(d_slot_src);
        if (d_diag_ptr) cudaFree(d_diag_ptr);
        if (d_diag_src) cudaFree(d_diag_src);
    }
    int upload() {
        if (d_slot_src) return GAPK_OK;
        auto up = [](void*& d, std::vector<int> const& v) -> cudaError_t {
            size_t bytes = (v.empty() ? 1 : v.size()) * sizeof(int);
            cudaError_t e = cudaMalloc(&d, bytes);
            if (e != cudaSuccess) return e;
            if (!v.empty()) e = cudaMemcpy(d, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice);
            return e;
        };
        cudaError_t e = up(d_slot_src, h.slot_src);
        if (e == cudaSuccess) e = up(d_diag_ptr, h.diag_ptr);
        if (e == cudaSuccess) e = up(d_diag_src, h.diag_src);
        if (e != cudaSuccess) {
            set_error(std::string("ybus upload: ") + cudaGetErrorString(e));
            return e == cudaErrorMemoryAllocation ? GAPK_ENOMEM : GAPK_ECUDA;
        }
        cudaGetDevice(&device);
        return GAPK_OK;
    }
};

// Branch results of solved scenarios: thread per (scenario, branch).  The stamps are the
// Y-bus builder's (same arithmetic, scaled to per unit), so the flows are those of the network
// the Newton loop solved.  out[(s * m + j) * 9 ..] = p_from, q_from, i_from, s_from, p_to,
// q_to, i_to, s_to, loading (W, var, A, VA); zeros for out-of-service branches (from < 0).
__global__ void k_branch_flows(int n_scen, int n_bus, int m, const int* __restrict__ from,
                               const int* __restrict__ to, const double* __restrict__ br,
                               int64_t branch_stride, const double2* __restrict__ v, double zb,
                               double base_power, double u_base, const double* __restrict__ i_n,
                               const double* __restrict__ sn, int mode, double* __restrict__ out) {
    const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (long)n_scen * m) return;
    const int s = (int)(tid / m), j = (int)(tid % m);
    double* o = out + (size_t)tid * 9;
    const int f = from[j], t = to[j];
    if (f < 0 || t < 0) {
        for (int c = 0; c < 9; ++c) o[c] = 0.0;
        return;
    }
    const Stamps st = branch_stamps(br + (size_t)s * branch_stride + (size_t)j * 6, mode);
    const double2 vf = v[(size_t)s * n_bus + f], vt = v[(size_t)s * n_bus + t];
    // currents into the branch at each end, per unit
    const double ifr = zb * (st.ff.x * vf.x - st.ff.y * vf.y + st.ft.x * vt.x - st.ft.y * vt.y);
    const double ifi = zb * (st.ff.x * vf.y + st.ff.y * vf.x + st.ft.x * vt.y + st.ft.y * vt.x);
    const double itr = zb * (st.tf.x * vf.x - st.tf.y * vf.y + st.tt.x * vt.x - st.tt.y * vt.y);
    const double iti = zb * (st.tf.x * vf.y + st.tf.y * vf.x + st.tt.x * vt.y + st.tt.y * vt.x);
    // S = V conj(I), in VA
    const double pf = (vf.x * ifr + vf.y * ifi) * base_power;
    const double qf = (vf.y * ifr - vf.x * ifi) * base_power;
    const double pt = (vt.x * itr + vt.y * iti) * base_power;
    const double qt = (vt.y * itr - vt.x * iti) * base_power;
    const double sf = hypot(pf, qf), stt = hypot(pt, qt);
    const double k3 = 1.7320508075688772 * u_base;  // sqrt(3) x line-to-line base voltage
    const double af = sf / (k3 * hypot(vf.x, vf.y)), at = stt / (k3 * hypot(vt.x, vt.y));
    double load = 0.0;
    if (i_n && i_n[j] > 0.0)
        load = fmax(af, at) / i_n[j];
    else if (sn && sn[j] > 0.0)
        load = fmax(sf, stt) / sn[j];
    o[0] = pf;
    o[1] = qf;
    o[2] = af;
    o[3] = sf;
    o[4] = pt;
    o[5] = qt;
    o[6] = at;
    o[7] = stt;
    o[8] = load;
}

extern "C" {

int gapk_ybus_create(int n_bus, int n_branch, const int* h_from_idx, const int* h_to_idx,
                     const int* h_in_service, int n_shunt, const int* h_shunt_bus,
                     gapk_ybus* out) {
    TraceRange tr("gapk_ybus_create: Y-bus pattern");
    if (!out || n_bus < 0 || n_branch < 0 || n_shunt < 0 ||
        (n_branch && (!h_from_idx || !h_to_idx || !h_in_service)) || (n_shunt && !h_shunt_bus)) {
        set_error("gapk_ybus_create: bad arguments");
        return GAPK_EINVAL;
    }
    auto y = std::make_unique<gapk_ybus_s>();
    build_ybus_pattern(n_bus, n_branch, h_from_idx, h_to_idx, h_in_service, n_shunt,
                       h_shunt_bus, y->h);
    *out = y.release();
    return GAPK_OK;
}

int gapk_ybus_destroy(gapk_ybus y) {
    delete y;
    return GAPK_OK;
}

int gapk_ybus_nnz(gapk_ybus y) { return y ? y->h.nnz : GAPK_EINVAL; }

int gapk_ybus_pattern(gapk_ybus y, int* h_row_ptr, int* h_col_idx) {
    if (!y || !h_row_ptr || (y->h.nnz && !h_col_idx)) {
        set_error("gapk_ybus_pattern: bad arguments");
        return GAPK_EINVAL;
    }
    std::copy(y->h.row_ptr.begin(), y->h.row_ptr.end(), h_row_ptr);
    std::copy(y->h.col_idx.begin(), y->h.col_idx.end(), h_col_idx);
    return GAPK_OK;
}

int gapk_ybus_assemble(gapk_ybus y, int n_scen, const double* d_branch, int64_t branch_stride,
                       const double* d_shunt, int64_t shunt_stride, int mode, double scale,
                       double* d_values, int64_t values_stride, void* stream) {
    TraceRange tr("gapk_ybus_assemble");
    if (!y || n_scen <= 0 || !d_values || (y->h.n_branch && !d_branch) ||
        (y->h.n_shunt && !d_shunt) || (mode != GAPK_YBUS_REFERENCE && mode != GAPK_YBUS_TAPS) ||
        branch_stride < 0 || shunt_stride < 0 || (n_scen > 1 && values_stride < y->h.nnz)) {
        set_error("gapk_ybus_assemble: bad arguments");
        return GAPK_EINVAL;
    }
    int rc = y->upload();
    if (rc) return rc;
    const long long total = (long long)y->h.nnz * n_scen;
    if (total == 0) return GAPK_OK;
    const int thr = 256;
    const unsigned blocks = static_cast<unsigned>((total + thr - 1) / thr);
    k_ybus<<<blocks, thr, 0, static_cast<cudaStream_t>(stream)>>>(
        y->h.nnz, n_scen, static_cast<const int*>(y->d_slot_src),
        static_cast<const int*>(y->d_diag_ptr), static_cast<const int*>(y->d_diag_src),
        d_branch, branch_stride, d_shunt, shunt_stride, mode, scale,
        reinterpret_cast<double2*>(d_values), values_stride);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("k_ybus launch: ") + cudaGetErrorString(e));
        return GAPK_ECUDA;
    }
    return GAPK_OK;
}

}  // extern "C"

// Segmented plan of branch changes: for every scenario, the CSR slots its changes touch, each
// with its (change, role) list in change order.
struct gapk_ybus_delta_s {
    int n_scen = 0, n_changes = 0;
    std::vector<int> items;  // int4 per (scenario, slot): scenario, slot, seg begin, seg end
    std::vector<int> seg;
    int device = -1;
    void* d_items = nullptr;
    void* d_seg = nullptr;
    ~gapk_ybus_delta_s() {
        if (d_items) cudaFree(d_items);
        if (d_seg) cudaFree(d_seg);
    }
    int upload() {
        if (d_items || items.empty()) return GAPK_OK;
        cudaError_t e = cudaMalloc(&d_items, items.size() * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&d_seg, std::max<size_t>(seg.size(), 1) * sizeof(int));
        if (e == cudaSuccess)
            e = cudaMemcpy(d_items, items.data(), items.size() * sizeof(int), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !seg.empty())
            e = cudaMemcpy(d_seg, seg.data(), seg.size() * sizeof(int), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            set_error(std::string("ybus delta upload: ") + cudaGetErrorString(e));
            return e == cudaErrorMemoryAllocation ? GAPK_ENOMEM : GAPK_ECUDA;
        }
        cudaGetDevice(&device);
        return GAPK_OK;
    }
};

namespace {

int delta_build(int n_scen, const int* change_ptr, const int* pos, gapk_ybus_delta_s& d) {
    d.n_scen = n_scen;
    d.n_changes = change_ptr[n_scen];
    std::vector<std::pair<int, int>> touch;  // (slot, change << 2 | role), per scenario
    for (int s = 0; s < n_scen; ++s) {
        if (change_ptr[s + 1] < change_ptr[s]) return GAPK_EINVAL;
        touch.clear();
        for (int c = change_ptr[s]; c < change_ptr[s + 1]; ++c)
            for (int r = 0; r < 4; ++r)
                if (pos[4 * c + r] >= 0) touch.emplace_back(pos[4 * c + r], c << 2 | r);
        // by slot; within a slot in change order (stable: the list is built in change order)
        std::stable_sort(touch.begin(), touch.end(),
                         [](auto const& a, auto const& b) { return a.first < b.first; });
        for (size_t i = 0; i < touch.size();) {
            size_t j = i;
            while (j < touch.size() && touch[j].first == touch[i].first) ++j;
            d.items.insert(d.items.end(), {s, touch[i].first, static_cast<int>(d.seg.size()),
                                           static_cast<int>(d.seg.size() + (j - i))});
            for (size_t k = i; k < j; ++k) d.seg.push_back(touch[k].second);
            i = j;
        }
    }
    return GAPK_OK;
}

int delta_launch(gapk_ybus_delta_s& d, const double* d_params, int mode, double scale,
                 double* d_values, int64_t stride, cudaStream_t st) {
    int rc = d.upload();
    if (rc) return rc;
    const int n_items = static_cast<int>(d.items.size() / 4);
    if (n_items == 0) return GAPK_OK;
    k_ybus_delta<<<(n_items + 255) / 256, 256, 0, st>>>(
        n_items, static_cast<const int4*>(d.d_items), static_cast<const int*>(d.d_seg), d_params,
        mode, scale, reinterpret_cast<double2*>(d_values), stride);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("k_ybus_delta launch: ") + cudaGetErrorString(e));
        return GAPK_ECUDA;
    }
    return GAPK_OK;
}

}  // namespace

extern "C" {

int gapk_ybus_delta_create(int n_scen, const int* h_change_ptr, const int* h_pos,
                           gapk_ybus_delta* out) {
    if (!out || n_scen <= 0 || !h_change_ptr || h_change_ptr[0] != 0 ||
        (h_change_ptr[n_scen] > 0 && !h_pos)) {
        set_error("gapk_ybus_delta_create: bad arguments");
        return GAPK_EINVAL;
    }
    auto d = std::make_unique<gapk_ybus_delta_s>();
    if (delta_build(n_scen, h_change_ptr, h_pos, *d)) {
        set_error("gapk_ybus_delta_create: change_ptr must be non-decreasing");
        return GAPK_EINVAL;
    }
    *out = d.release();
    return GAPK_OK;
}

int gapk_ybus_delta_destroy(gapk_ybus_delta d) {
    delete d;
    return GAPK_OK;
}

int gapk_ybus_delta_apply(gapk_ybus_delta d, const double* d_params, int mode, double scale,
                          double* d_values, int64_t values_stride, void* stream) {
    if (!d || !d_values ||
        (mode != GAPK_DELTA_REFERENCE && mode != GAPK_DELTA_FIXED &&
         mode != GAPK_DELTA_FIXED_TAPS) ||
        (d->n_changes > 0 && !d_params) || (d->n_scen > 1 && values_stride <= 0)) {
        set_error("gapk_ybus_delta_apply: bad arguments");
        return GAPK_EINVAL;
    }
    return delta_launch(*d, d_params, mode, scale, d_values, values_stride,
                        static_cast<cudaStream_t>(stream));
}

int gapk_ybus_apply_changes(int n_changes, const int* h_pos, const double* d_params, int mode,
                            double* d_values, void* stream) {
    if (n_changes < 0 || (n_changes > 0 && (!h_pos || !d_params || !d_values))) {
        set_error("gapk_ybus_apply_changes: bad arguments");
        return GAPK_EINVAL;
    }
    if (n_changes == 0) return GAPK_OK;
    const int ptr[2] = {0, n_changes};
    gapk_ybus_delta_s d;
    if (delta_build(1, ptr, h_pos, d)) return GAPK_EINVAL;
    return gapk_ybus_delta_apply(&d, d_params, mode, 1.0, d_values, 0, stream);
}

int gapk_branch_flows(int n_scen, int n_bus, int n_branch, const int* d_from, const int* d_to,
                      const double* d_branch, int64_t branch_stride, const double* d_v,
                      double base_power, double u_base, const double* d_i_n, const double* d_sn,
                      int mode, double* d_out, void* stream) {
    if (n_scen <= 0 || n_bus <= 0 || n_branch < 0 || base_power <= 0.0 || u_base <= 0.0 ||
        (n_branch && (!d_from || !d_to || !d_branch || !d_v || !d_out)) || branch_stride < 0 ||
        (n_scen > 1 && branch_stride != 0 && branch_stride < (int64_t)n_branch * 6) ||
        (mode != GAPK_YBUS_REFERENCE && mode != GAPK_YBUS_TAPS)) {
        set_error("gapk_branch_flows: bad arguments");
        return GAPK_EINVAL;
    }
    if (n_branch == 0) return GAPK_OK;
    const long total = (long)n_scen * n_branch;
    const double zb = u_base * u_base / base_power;
    k_branch_flows<<<(unsigned)((total + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        n_scen, n_bus, n_branch, d_from, d_to, d_branch, branch_stride,
        reinterpret_cast<const double2*>(d_v), zb, base_power, u_base, d_i_n, d_sn, mode, d_out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("k_branch_flows launch: ") + cudaGetErrorString(e));
        return GAPK_ECUDA;
    }
    return GAPK_OK;
}

}  // extern "C"
