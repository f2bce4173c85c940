// libgap_admittance_gpu.so -- IAdmittanceMatrix on the B200 engine.
//
// Replaces src/admittance/gpu/gpu_admittance_matrix.cu (factory at :577-585).  The CSR
// pattern is the reference CPU builder's (stable-sorted triplets, duplicates kept) and the
// values come from the device's deterministic segmented reduction, bit-identical to
// src/admittance/cpu/cpu_admittance_matrix.cpp:44-202.  Transformer taps and phase shifts
// are ignored, as the reference does, unless GAP_B200_YBUS_TAPS=1 is set in the environment.
#include <algorithm>
#include <cstdlib>

#include "common.hpp"

namespace gapb200 {

class B200AdmittanceMatrix final : public gap::admittance::IAdmittanceMatrix {
  public:
    ~B200AdmittanceMatrix() override {
        if (ybus_) gapk_ybus_destroy(ybus_);
    }

    std::unique_ptr<gap::SparseMatrix> build_admittance_matrix(
        gap::NetworkData const& net) override {
        const int n = static_cast<int>(net.buses.size());
        int max_id = -1;
        auto lut = id_to_index(net, max_id);
        auto look = [&](int id) { return (id >= 0 && id <= max_id) ? lut[id] : -1; };
        const int m = static_cast<int>(net.branches.size());
        std::vector<int> f(m), t(m), valid(m);
        std::vector<double> prm(static_cast<size_t>(m) * 6);
        for (int b = 0; b < m; ++b) {
            auto const& br = net.branches[b];
            int fi = look(br.from_bus), ti = look(br.to_bus);
            bool ok = br.status && fi >= 0 && fi < n && ti >= 0 && ti < n;
            f[b] = ok ? fi : 0;
            t[b] = ok ? ti : 0;
            valid[b] = ok ? 1 : 0;
            double* q = &prm[static_cast<size_t>(b) * 6];
            q[0] = br.r1;
            q[1] = br.x1;
            q[2] = br.g1;
            q[3] = br.b1;
            q[4] = br.k;
            q[5] = br.theta;
        }
        std::vector<int> sb;
        std::vector<double> sh;
        for (auto const& a : net.appliances) {
            if (a.type != gap::ApplianceType::SHUNT) continue;
            int bi = look(a.node);
            if (bi < 0 || bi >= n) continue;
            sb.push_back(bi);
            sh.push_back(a.g1);
            sh.push_back(a.b1);
        }
        if (!ybus_ || n != n_ || f != f_ || t != t_ || valid != valid_ || sb != sb_) {
            if (ybus_) gapk_ybus_destroy(ybus_);
            ybus_ = nullptr;
            check(gapk_ybus_create(n, m, f.data(), t.data(), valid.data(),
                                   static_cast<int>(sb.size()), sb.data(), &ybus_),
                  "gapk_ybus_create");
            n_ = n;
            f_ = f;
            t_ = t;
            valid_ = valid;
            sb_ = sb;
        }
        auto Y = std::make_unique<gap::SparseMatrix>();
        Y->num_rows = Y->num_cols = n;
        Y->nnz = gapk_ybus_nnz(ybus_);
        Y->row_ptr.resize(n + 1);
        Y->col_idx.resize(Y->nnz);
        check(gapk_ybus_pattern(ybus_, Y->row_ptr.data(), Y->col_idx.data()), "gapk_ybus_pattern");
        if (sh.empty()) sh.assign(2, 0.0);
        double* dp = d_branch_.upload(prm);
        double* ds = d_shunt_.upload(sh);
        double* dv = static_cast<double*>(d_values_.ensure(static_cast<size_t>(Y->nnz) * 16));
        const char* env = std::getenv("GAP_B200_YBUS_TAPS");
        const int mode = (env && std::atoi(env) != 0) ? GAPK_YBUS_TAPS : GAPK_YBUS_REFERENCE;
        check(gapk_ybus_assemble(ybus_, 1, dp, 0, ds, 0, mode, 1.0, dv, Y->nnz, nullptr),
              "gapk_ybus_assemble");
        Y->values.resize(Y->nnz);
        check_cuda(cudaMemcpy(Y->values.data(), dv, static_cast<size_t>(Y->nnz) * 16,
                              cudaMemcpyDeviceToHost),
                   "cudaMemcpy D2H");
        return Y;
    }

    // Reference semantics (src/admittance/cpu/cpu_admittance_matrix.cpp:204-301): branch
    // endpoints are taken as matrix indices (shifted down by one when both are positive and
    // one exceeds the matrix size); the first matching CSR entries are updated.  The value
    // arithmetic runs on the device, one thread per touched entry, each entry's changes in
    // change order.  By default the reference's own update, bit for bit (its diagonal delta
    // carries j b1 + j b1/2, unlike its build); GAP_B200_YBUS_UPDATE=fixed applies the
    // builder's stamps instead, so that update(build(net)) equals build(changed net).
    std::unique_ptr<gap::SparseMatrix> update_admittance_matrix(
        gap::SparseMatrix const& matrix, std::vector<gap::BranchData> const& changes) override {
        auto Y = std::make_unique<gap::SparseMatrix>(matrix);
        const int nr = Y->num_rows;
        std::vector<int> pos;
        std::vector<double> prm;
        auto find = [&](int r, int c) {
            for (int p = Y->row_ptr[r]; p < Y->row_ptr[r + 1]; ++p)
                if (Y->col_idx[p] == c) return p;
            return -1;
        };
        for (auto const& ch : changes) {
            int f = ch.from_bus, t = ch.to_bus;
            if (f > 0 && t > 0 && (f > nr || t > nr)) {
                f -= 1;
                t -= 1;
            }
            if (f < 0 || f >= nr || t < 0 || t >= nr) continue;
            pos.insert(pos.end(), {find(f, f), find(t, t), find(f, t), find(t, f)});
            prm.insert(prm.end(), {ch.r1, ch.x1, ch.g1, ch.b1, 1.0, 0.0, ch.status ? 1.0 : 0.0});
        }
        if (pos.empty() || Y->values.empty()) return Y;
        const char* env = std::getenv("GAP_B200_YBUS_UPDATE");
        const int mode = (env && std::string(env) == "fixed") ? GAPK_DELTA_FIXED
                                                              : GAPK_DELTA_REFERENCE;
        double* dprm = d_branch_.upload(prm);
        double* dv = static_cast<double*>(d_values_.ensure(Y->values.size() * 16));
        check_cuda(cudaMemcpy(dv, Y->values.data(), Y->values.size() * 16, cudaMemcpyHostToDevice),
                   "cudaMemcpy H2D");
        check(gapk_ybus_apply_changes(static_cast<int>(pos.size() / 4), pos.data(), dprm, mode, dv,
                                      nullptr),
              "gapk_ybus_apply_changes");
        check_cuda(cudaMemcpy(Y->values.data(), dv, Y->values.size() * 16, cudaMemcpyDeviceToHost),
                   "cudaMemcpy D2H");
        return Y;
    }

    gap::BackendType get_backend_type() const noexcept override {
        return gap::BackendType::GPU_CUDA;
    }

  private:
    gapk_ybus ybus_ = nullptr;
    int n_ = -1;
    std::vector<int> f_, t_, valid_, sb_;
    DeviceBuffer d_branch_, d_shunt_, d_values_;
};

}  // namespace gapb200

extern "C" {
gap::admittance::IAdmittanceMatrix* create_gpu_admittance_matrix() {
    return new gapb200::B200AdmittanceMatrix();
}
void destroy_gpu_admittance_matrix(gap::admittance::IAdmittanceMatrix* instance) {
    delete instance;
}
}
