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

#include <memory>
#include <string>
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

// Branch status changes applied to existing values, in change order (one thread: the deltas
// of different changes may hit the same entry, and the reference applies them sequentially,
// src/admittance/cpu/cpu_admittance_matrix.cpp:214-297).  pos = (diag f, diag t, (f,t), (t,f))
// CSR indices or -1; prm = (r1, x1, g1, b1, status).
__global__ void k_ybus_changes(int n, const int* __restrict__ pos, const double* __restrict__ prm,
                               double2* values) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int i = 0; i < n; ++i) {
        const double* q = prm + (size_t)i * 5;
        const double r = q[0], x = q[1], g = q[2], b = q[3];
        const double z2 = __dadd_rn(__dmul_rn(r, r), __dmul_rn(x, x));
        double yr = 0.0, yi = 0.0;
        if (z2 > 1e-12) {
            yr = __ddiv_rn(r, z2);
            yi = __ddiv_rn(-x, z2);
        }
        // total = series + (g1 + j b1); the diagonals also get j b1/2 (the reference's
        // update adds both, unlike its build)
        double tr = __dadd_rn(yr, g), ti = __dadd_rn(yi, b);
        double sr = 0.0, si = __ddiv_rn(b, 2.0);
        double orr = yr, oi = yi;
        if (q[4] == 0.0) {
            tr = -tr;
            ti = -ti;
            si = -si;
            orr = -orr;
            oi = -oi;
            sr = -sr;
        }
        const double dr = __dadd_rn(tr, sr), di = __dadd_rn(ti, si);
        const int* p = pos + (size_t)i * 4;
        for (int k = 0; k < 2; ++k)
            if (p[k] >= 0) {
                double2 v = values[p[k]];
                values[p[k]] = make_double2(__dadd_rn(v.x, dr), __dadd_rn(v.y, di));
            }
        for (int k = 2; k < 4; ++k)
            if (p[k] >= 0) {
                double2 v = values[p[k]];
                values[p[k]] = make_double2(__dsub_rn(v.x, orr), __dsub_rn(v.y, oi));
            }
    }
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

int gapk_ybus_apply_changes(int n_changes, const int* d_pos, const double* d_params,
                            double* d_values, void* stream) {
    if (n_changes < 0 || (n_changes > 0 && (!d_pos || !d_params || !d_values))) {
        set_error("gapk_ybus_apply_changes: bad arguments");
        return GAPK_EINVAL;
    }
    if (n_changes == 0) return GAPK_OK;
    k_ybus_changes<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(
        n_changes, d_pos, d_params, reinterpret_cast<double2*>(d_values));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("k_ybus_changes launch: ") + cudaGetErrorString(e));
        return GAPK_ECUDA;
    }
    return GAPK_OK;
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
