// libgap_lu_gpu.so -- ILUSolver on the B200 engine's general sparse LU.
//
// Replaces src/solver/lu/gpu/gpu_cudss_solver.cu (factories at :489-497) and
// src/solver/lu/gpu/gpu_lu_solver.cu (:203-207).  Analysis is cached per sparsity pattern
// (zero-free-diagonal row matching, minimum-degree ordering, symbolic factorisation on the
// host); factorisation and solves run on the device with static pivoting.  Error behaviour
// follows CPULUSolver (src/solver/lu/cpu/cpu_lu_solver.cpp:91-185): factorize() returns false
// for non-square, empty or numerically singular matrices; solve() throws before a successful
// factorisation or on a right-hand side of the wrong size.
#include "common.hpp"

namespace gapb200 {

class B200LUSolver final : public gap::solver::ILUSolver {
  public:
    ~B200LUSolver() override {
        if (lu_) gapk_splu_destroy(lu_);
    }

    bool factorize(gap::SparseMatrix const& m) override {
        factorized_ = false;
        if (m.num_rows != m.num_cols || m.nnz <= 0 || m.values.empty()) return false;
        if (static_cast<int>(m.row_ptr.size()) != m.num_rows + 1 ||
            static_cast<int>(m.col_idx.size()) < m.nnz || static_cast<int>(m.values.size()) < m.nnz)
            return false;
        if (!lu_ || m.num_rows != n_ || m.row_ptr != rp_ ||
            !std::equal(m.col_idx.begin(), m.col_idx.begin() + m.nnz, ci_.begin(), ci_.end())) {
            if (lu_) gapk_splu_destroy(lu_);
            lu_ = nullptr;
            if (gapk_splu_create(m.num_rows, m.nnz, m.row_ptr.data(), m.col_idx.data(), &lu_) !=
                GAPK_OK)
                return false;
            n_ = m.num_rows;
            rp_ = m.row_ptr;
            ci_.assign(m.col_idx.begin(), m.col_idx.begin() + m.nnz);
        }
        void* dv = d_values_.ensure(static_cast<size_t>(m.nnz) * 16);
        check_cuda(cudaMemcpy(dv, m.values.data(), static_cast<size_t>(m.nnz) * 16,
                              cudaMemcpyHostToDevice),
                   "cudaMemcpy H2D");
        int rc = gapk_splu_factorize(lu_, static_cast<const double*>(dv), nullptr);
        if (rc == GAPK_ESINGULAR) return false;
        check(rc, "gapk_splu_factorize");
        factorized_ = true;
        return true;
    }

    gap::ComplexVector solve(gap::ComplexVector const& rhs) override {
        if (!factorized_) throw std::runtime_error("Matrix not factorized. Call factorize() first.");
        if (static_cast<int>(rhs.size()) != n_)
            throw std::runtime_error("RHS size does not match matrix dimension");
        void* db = d_rhs_.ensure(rhs.size() * 16);
        void* dx = d_x_.ensure(rhs.size() * 16);
        check_cuda(cudaMemcpy(db, rhs.data(), rhs.size() * 16, cudaMemcpyHostToDevice),
                   "cudaMemcpy H2D");
        check(gapk_splu_solve(lu_, static_cast<const double*>(db), static_cast<double*>(dx), nullptr),
              "gapk_splu_solve");
        gap::ComplexVector x(rhs.size());
        check_cuda(cudaMemcpy(x.data(), dx, rhs.size() * 16, cudaMemcpyDeviceToHost),
                   "cudaMemcpy D2H");
        return x;
    }

    bool update_factorization(gap::SparseMatrix const& m) override { return factorize(m); }
    gap::BackendType get_backend_type() const noexcept override {
        return gap::BackendType::GPU_CUDA;
    }
    bool is_factorized() const noexcept override { return factorized_; }

  private:
    gapk_splu lu_ = nullptr;
    int n_ = -1;
    std::vector<int> rp_, ci_;
    bool factorized_ = false;
    DeviceBuffer d_values_, d_rhs_, d_x_;
};

}  // namespace gapb200

extern "C" {
gap::solver::ILUSolver* create_gpu_lu_solver() { return new gapb200::B200LUSolver(); }
void destroy_gpu_lu_solver(gap::solver::ILUSolver* instance) { delete instance; }
gap::solver::ILUSolver* create_gpu_ilu_solver() { return new gapb200::B200LUSolver(); }
void destroy_gpu_ilu_solver(gap::solver::ILUSolver* instance) { delete instance; }
}
