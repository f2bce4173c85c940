// Internal declarations shared by the host analysis (symbolic.cpp) and the device code.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace gapk {

void set_error(std::string const& msg);

// NVTX range over a host call (plan analysis, batch set-up, solve enqueue, stages), so that a
// profiler's timeline names the engine's phases; without a tool attached a push/pop costs a few
// nanoseconds.  Defined in nr.cu (NVTX v3, header only).
struct TraceRange {
    explicit TraceRange(const char* name);
    ~TraceRange();
    TraceRange(TraceRange const&) = delete;
    TraceRange& operator=(TraceRange const&) = delete;
};

// ---- Y-bus pattern -------------------------------------------------------------------
// Source encoding of one CSR slot:
//   off-diagonal triplet of branch b in direction d (0: (from,to), 1: (to,from)) -> 2*b + d
//   the diagonal triplet of bus i                                           -> -(i + 1)
// Diagonal contributions of bus i, in the reference's accumulation order, are listed in
// diag_src[diag_ptr[i] .. diag_ptr[i+1]):
//   branch end: 2*b + side (0: from end, 1: to end);  shunt s: -(s + 1)
struct YbusPatternHost {
    int n_bus = 0, n_branch = 0, n_shunt = 0, nnz = 0;
    std::vector<int> row_ptr, col_idx, slot_src, diag_ptr, diag_src;
};

void build_ybus_pattern(int n_bus, int n_branch, const int* from, const int* to,
                        const int* in_service, int n_shunt, const int* shunt_bus,
                        YbusPatternHost& out);

// ---- Newton-Raphson symbolic analysis ------------------------------------------------
// Block unknowns ("nodes") are the non-slack buses numbered in elimination order.  Each node
// carries a 2x2 block: rows (P, Q) x columns (theta, |V|).  PV buses keep the block shape;
// their Q row and |V| column are a decoupled identity (rhs 0, solution 0).
//
// Factor storage, one 2x2 block per slot:
//   slot k                      : D_k, holding D_k^-1 after factorisation (k < nb)
//   slot nb + p                 : L(lidx[p], k) for p in [lptr[k], lptr[k+1])
//   slot nb + nnz_l + p         : U(k, lidx[p])
struct NRPlanHost {
    int n_bus = 0, nb = 0, n_pq = 0, n_pv = 0, n_slack = 0, n_vars = 0, nnz_y = 0;
    int nnz_l = 0, n_slots = 0, n_levels = 0, max_level_width = 0;
    int jac_mode = 0;
    std::vector<int> bus_type;
    std::vector<int> node_of_bus, bus_of_node, node_pq;
    std::vector<int> lptr, lidx;
    std::vector<int> level_ptr, level_nodes, node_level;
    // Jacobian fill: per slot (row_bus, col_bus, src_begin, src_end); sources index the Y CSR
    std::vector<int> slot_info, slot_src;
    // blocks of the Jacobian pattern itself ("A blocks"), by block row, for residuals:
    // arow_ptr[nb+1], arow (a_slot, col_node) pairs
    std::vector<int> arow_ptr, arow;
    std::vector<int> slot_a;  // A index of each slot, -1 for fill-only slots
    std::vector<int> a_slots;  // slot of each A block (inverse of slot_a)
    std::vector<int> acol_ptr, acol;  // A blocks by block column: (a index, row node) pairs
    int n_a = 0;
    // numeric factorisation schedule
    //   level h, phase A: targets [fa_ptr[h], fa_ptr[h+1]) = (slot, pair_begin, pair_end, flags)
    //     flags bit 0: diagonal slot (inverted); bit 1: slot holds a Jacobian value
    //   level h, phase B: scale   [fb_ptr[h], fb_ptr[h+1]) = (L slot, D slot)
    std::vector<int> fa_ptr, targets, fb_ptr, scale;
    std::vector<int> pairs;  // (left slot, right slot)
    int64_t n_pairs = 0;
    // dense tail: the last n_tail nodes (ns = nb - n_tail sparse nodes before them);
    // schur[4*t..] = (slot, pair_begin, pair_end, block position r*n_tail + c | hasval << 30)
    int n_tail = 0, ns = 0;
    std::vector<int> schur;
    // forward solve row lists: for node k, (L slot, node m) pairs over sparse m, k in struct(m)
    std::vector<int> rptr, rlist;
    // reference variable order <-> node components: var_of[node*2+c] = reference index or -1
    std::vector<int> var_of_comp;
    // reference equation order: eq_of_comp[node*2+c]
    std::vector<int> eq_of_comp;
};

bool analyze_nr(int n_bus, int nnz_y, const int* y_row_ptr, const int* y_col_idx,
                const int* bus_type, int jac_mode, int ordering, int dense_min, NRPlanHost& out);

// General square sparse matrix (complex values handled as 2x2 real blocks by the caller):
// a zero-free-diagonal row permutation rp, then the same analysis as the Newton plan on the
// permuted pattern (every position an unknown, duplicate entries summed).  val_map[e] maps
// entry e of the permuted CSR (the plan's "Y") back to the caller's entry index.
bool analyze_general(int n, int nnz, const int* row_ptr, const int* col_idx, int dense_min,
                     NRPlanHost& P, std::vector<int>& rp, std::vector<int>& val_map);

}  // namespace gapk
