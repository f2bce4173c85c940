// Host-side analysis, run once per topology:
//   * the Y-bus CSR pattern in the reference's triplet order
//     (src/admittance/cpu/cpu_admittance_matrix.cpp:100-186), with per-slot sources and the
//     per-bus diagonal contribution lists for the device's segmented reduction;
//   * the Newton-Raphson plan: 2x2-block Jacobian pattern on the non-slack buses, a
//     minimum-degree elimination order, the symbolic block factorisation (elimination graph),
//     the elimination-tree level schedule and all index lists the device kernels walk.
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <set>
#include <stdexcept>
#include <utility>

#include "internal.h"

namespace gapk {

void build_ybus_pattern(int n_bus, int n_branch, const int* from, const int* to,
                        const int* in_service, int n_shunt, const int* shunt_bus,
                        YbusPatternHost& out) {
    struct Trip {
        int row, col, src;
    };
    std::vector<Trip> trips;
    trips.reserve(static_cast<size_t>(n_bus) + 2 * static_cast<size_t>(n_branch));
    auto valid = [&](int b) {
        return in_service[b] != 0 && from[b] >= 0 && from[b] < n_bus && to[b] >= 0 &&
               to[b] < n_bus;
    };
    // off-diagonal triplets in branch order (cpu_admittance_matrix.cpp:138-139)
    for (int b = 0; b < n_branch; ++b) {
        if (!valid(b)) continue;
        trips.push_back({from[b], to[b], 2 * b});
        trips.push_back({to[b], from[b], 2 * b + 1});
    }
    // diagonal triplets last (cpu_admittance_matrix.cpp:143-145)
    for (int i = 0; i < n_bus; ++i) trips.push_back({i, i, -(i + 1)});
    std::stable_sort(trips.begin(), trips.end(), [](Trip const& a, Trip const& b) {
        if (a.row != b.row) return a.row < b.row;
        return a.col < b.col;
    });
    out.n_bus = n_bus;
    out.n_branch = n_branch;
    out.n_shunt = n_shunt;
    out.nnz = static_cast<int>(trips.size());
    out.row_ptr.assign(n_bus + 1, 0);
    out.col_idx.resize(trips.size());
    out.slot_src.resize(trips.size());
    for (size_t p = 0; p < trips.size(); ++p) {
        out.row_ptr[trips[p].row + 1]++;
        out.col_idx[p] = trips[p].col;
        out.slot_src[p] = trips[p].src;
    }
    for (int i = 0; i < n_bus; ++i) out.row_ptr[i + 1] += out.row_ptr[i];
    // diagonal accumulation order: shunts (appliance order, :88-97), then branch ends in branch
    // order, from end before to end (:134-135)
    std::vector<int> cnt(n_bus + 1, 0);
    for (int s = 0; s < n_shunt; ++s)
        if (shunt_bus[s] >= 0 && shunt_bus[s] < n_bus) cnt[shunt_bus[s] + 1]++;
    for (int b = 0; b < n_branch; ++b) {
        if (!valid(b)) continue;
        cnt[from[b] + 1]++;
        cnt[to[b] + 1]++;
    }
    for (int i = 0; i < n_bus; ++i) cnt[i + 1] += cnt[i];
    out.diag_ptr = cnt;
    out.diag_src.assign(cnt[n_bus], 0);
    std::vector<int> fillp(cnt.begin(), cnt.end() - 1);
    for (int s = 0; s < n_shunt; ++s)
        if (shunt_bus[s] >= 0 && shunt_bus[s] < n_bus) out.diag_src[fillp[shunt_bus[s]]++] = -(s + 1);
    for (int b = 0; b < n_branch; ++b) {
        if (!valid(b)) continue;
        out.diag_src[fillp[from[b]]++] = 2 * b;
        out.diag_src[fillp[to[b]]++] = 2 * b + 1;
    }
}

namespace {

// Elimination on the quotient-free elimination graph.  Returns the elimination order (as
// indices into the node list) and, per eliminated node, its neighbour set at elimination
// (= the strictly-lower structure of its column of L).  Minimum degree, ties broken by the
// lower index, so the result is deterministic.
void eliminate(int nq, std::vector<std::vector<int>>& adj, bool mindeg, std::vector<int>& order,
               std::vector<std::vector<int>>& structq) {
    order.clear();
    order.reserve(nq);
    structq.assign(nq, {});
    std::vector<char> done(nq, 0);
    std::set<std::pair<int, int>> pq;
    if (mindeg)
        for (int q = 0; q < nq; ++q) pq.insert({static_cast<int>(adj[q].size()), q});
    std::vector<int> tmp;
    for (int step = 0; step < nq; ++step) {
        int v;
        if (mindeg) {
            v = pq.begin()->second;
            pq.erase(pq.begin());
        } else {
            v = step;
        }
        done[v] = 1;
        order.push_back(v);
        std::vector<int> nbrs = std::move(adj[v]);
        adj[v].clear();
        for (int u : nbrs) {
            if (mindeg) pq.erase({static_cast<int>(adj[u].size()), u});
            tmp.clear();
            std::set_union(adj[u].begin(), adj[u].end(), nbrs.begin(), nbrs.end(),
                           std::back_inserter(tmp));
            adj[u].clear();
            for (int w : tmp)
                if (w != u && w != v) adj[u].push_back(w);
            if (mindeg) pq.insert({static_cast<int>(adj[u].size()), u});
        }
        structq[v] = std::move(nbrs);
    }
}

inline int find_in(std::vector<int> const& lidx, int b, int e, int x) {
    auto it = std::lower_bound(lidx.begin() + b, lidx.begin() + e, x);
    if (it == lidx.begin() + e || *it != x) return -1;
    return static_cast<int>(it - lidx.begin());
}

}  // namespace

bool analyze_nr(int n_bus, int nnz_y, const int* y_row_ptr, const int* y_col_idx,
                const int* bus_type, int jac_mode, int ordering, int dense_min, NRPlanHost& P) {
    P = NRPlanHost{};
    P.n_bus = n_bus;
    P.nnz_y = nnz_y;
    P.jac_mode = jac_mode;
    P.bus_type.assign(bus_type, bus_type + n_bus);
    if (y_row_ptr[0] != 0 || y_row_ptr[n_bus] != nnz_y) {
        set_error("Y row_ptr inconsistent with nnz");
        return false;
    }
    for (int i = 0; i < n_bus; ++i) {
        if (y_row_ptr[i + 1] < y_row_ptr[i]) {
            set_error("Y row_ptr not monotone");
            return false;
        }
        int t = bus_type[i];
        if (t < 0 || t > 2) {
            set_error("bus_type must be 0 (PQ), 1 (PV) or 2 (SLACK)");
            return false;
        }
        if (t == 2) P.n_slack++;
        if (t == 1) P.n_pv++;
        if (t == 0) P.n_pq++;
    }
    for (int p = 0; p < nnz_y; ++p) {
        if (y_col_idx[p] < 0 || y_col_idx[p] >= n_bus) {
            set_error("Y col_idx out of range");
            return false;
        }
    }
    P.n_vars = (n_bus - P.n_slack) + P.n_pq;

    // node candidates: non-slack buses in bus order (q index)
    std::vector<int> q_of_bus(n_bus, -1), bus_of_q;
    for (int i = 0; i < n_bus; ++i)
        if (bus_type[i] != 2) {
            q_of_bus[i] = static_cast<int>(bus_of_q.size());
            bus_of_q.push_back(i);
        }
    const int nb = static_cast<int>(bus_of_q.size());
    P.nb = nb;

    // symmetrised block graph
    std::vector<std::vector<int>> adj(nb);
    for (int i = 0; i < n_bus; ++i) {
        int qi = q_of_bus[i];
        if (qi < 0) continue;
        for (int p = y_row_ptr[i]; p < y_row_ptr[i + 1]; ++p) {
            int qj = q_of_bus[y_col_idx[p]];
            if (qj < 0 || qj == qi) continue;
            adj[qi].push_back(qj);
            adj[qj].push_back(qi);
        }
    }
    for (auto& a : adj) {
        std::sort(a.begin(), a.end());
        a.erase(std::unique(a.begin(), a.end()), a.end());
    }

    std::vector<int> order;
    std::vector<std::vector<int>> structq;
    eliminate(nb, adj, ordering == 0, order, structq);

    std::vector<int> node_of_q(nb);
    for (int k = 0; k < nb; ++k) node_of_q[order[k]] = k;
    P.node_of_bus.assign(n_bus, -1);
    P.bus_of_node.resize(nb);
    P.node_pq.resize(nb);
    for (int k = 0; k < nb; ++k) {
        int bus = bus_of_q[order[k]];
        P.bus_of_node[k] = bus;
        P.node_of_bus[bus] = k;
        P.node_pq[k] = bus_type[bus] == 0 ? 1 : 0;
    }
    // column structures
    P.lptr.assign(nb + 1, 0);
    for (int k = 0; k < nb; ++k) P.lptr[k + 1] = P.lptr[k] + static_cast<int>(structq[order[k]].size());
    P.nnz_l = P.lptr[nb];
    P.lidx.resize(P.nnz_l);
    for (int k = 0; k < nb; ++k) {
        auto& s = structq[order[k]];
        int b = P.lptr[k];
        for (size_t t = 0; t < s.size(); ++t) P.lidx[b + t] = node_of_q[s[t]];
        std::sort(P.lidx.begin() + b, P.lidx.begin() + P.lptr[k + 1]);
    }
    structq.clear();
    const int nnzl = P.nnz_l;
    P.n_slots = nb + 2 * nnzl;
    const int Lbase = nb, Ubase = nb + nnzl;

    // ---- dense trailing block ----
    // T = the longest run of trailing nodes whose columns are completely full
    // (struct(k) = {k+1, ..., nb-1}).  When T >= dense_min those nodes are factorised as one
    // dense 2T x 2T matrix per scenario; everything before them ("sparse part", ns nodes) is
    // factorised block by block on the level schedule.
    int T = 0;
    for (int k = nb - 1; k >= 0; --k) {
        if (P.lptr[k + 1] - P.lptr[k] == nb - 1 - k)
            ++T;
        else
            break;
    }
    if (dense_min <= 0 || T < dense_min) T = 0;
    if (T > 0) {
        // Extend the tail over the nodes just before it when that is cheaper: every extra
        // node grows the dense LU (~N^3) and the dense solves (~N^2) but removes the outer
        // products its column would add to the Schur gather (t_m^2 block pairs for a sparse
        // node with t_m tail neighbours) -- the last sparse nodes before a min-degree tail are
        // adjacent to most of it.  Costs per scenario in seconds, from B200 FP32 timings of
        // the kernels: dense LU 2/3 N^3 flops at 18.5 TFLOP/s, 2.7 ps per Schur pair, two
        // dense solves at 0.43 us per 466^2 entries.
        const int T0 = T, ns0 = nb - T0;
        const int kmax = std::min(ns0, 128);
        auto cost = [&](int kk) {
            const int nsk = ns0 - kk;
            double pairs = 0.0;
            for (int m = 0; m < nsk; ++m) {
                const int* b = P.lidx.data() + P.lptr[m];
                const int* e = P.lidx.data() + P.lptr[m + 1];
                const double t = static_cast<double>(e - std::lower_bound(b, e, nsk));
                pairs += t * t;
            }
            const double N = 2.0 * (T0 + kk);
            return (2.0 / 3.0) * N * N * N / 18.5e12 + 2.72e-12 * pairs +
                   8.6e-7 * (N / 466.0) * (N / 466.0);
        };
        double best = cost(0);
        for (int kk = 4; kk <= kmax; kk += 4) {
            const double c = cost(kk);
            if (c < best) {
                best = c;
                T = T0 + kk;
            }
        }
    }
    const int ns = nb - T;
    P.n_tail = T;
    P.ns = ns;

    // elimination-forest heights of the sparse nodes -> levels
    std::vector<int> height(ns, 0);
    for (int k = 0; k < ns; ++k) {
        if (P.lptr[k + 1] > P.lptr[k]) {
            int parent = P.lidx[P.lptr[k]];
            if (parent < ns) height[parent] = std::max(height[parent], height[k] + 1);
        }
    }
    int nlev = ns ? (*std::max_element(height.begin(), height.end()) + 1) : 0;
    P.n_levels = nlev;
    P.node_level = height;
    P.level_ptr.assign(nlev + 1, 0);
    for (int k = 0; k < ns; ++k) P.level_ptr[height[k] + 1]++;
    for (int h = 0; h < nlev; ++h) {
        P.max_level_width = std::max(P.max_level_width, P.level_ptr[h + 1]);
        P.level_ptr[h + 1] += P.level_ptr[h];
    }
    P.level_nodes.resize(ns);
    {
        std::vector<int> fp(P.level_ptr.begin(), P.level_ptr.end() - 1);
        for (int k = 0; k < ns; ++k) P.level_nodes[fp[height[k]]++] = k;
    }
    // Renumber the sparse nodes level by level (stable within a level).  Children have lower
    // heights than their parents, so this is another topological order of the same elimination
    // tree: the same fill, the same parents (a column's first entry), with the nodes of one
    // level contiguous, so that the level-scheduled kernels read their right-hand sides,
    // solutions, pivots and column pointers as contiguous runs.  The tail keeps its numbers.
    if (ns > 0) {
        std::vector<int> newk(nb);
        for (int t = 0; t < ns; ++t) newk[P.level_nodes[t]] = t;
        for (int k = ns; k < nb; ++k) newk[k] = k;
        std::vector<int> bus_of_node(nb), node_pq(nb), lptr(nb + 1, 0), lidx(P.nnz_l), lev(ns);
        for (int k = 0; k < nb; ++k) {
            const int k2 = newk[k];
            bus_of_node[k2] = P.bus_of_node[k];
            node_pq[k2] = P.node_pq[k];
            lptr[k2 + 1] = P.lptr[k + 1] - P.lptr[k];
        }
        for (int k = 0; k < nb; ++k) lptr[k + 1] += lptr[k];
        for (int k = 0; k < nb; ++k) {
            const int k2 = newk[k];
            int w = lptr[k2];
            for (int p = P.lptr[k]; p < P.lptr[k + 1]; ++p) lidx[w++] = newk[P.lidx[p]];
            std::sort(lidx.begin() + lptr[k2], lidx.begin() + lptr[k2 + 1]);
        }
        for (int k = 0; k < ns; ++k) lev[newk[k]] = height[k];
        P.bus_of_node.swap(bus_of_node);
        P.node_pq.swap(node_pq);
        P.lptr.swap(lptr);
        P.lidx.swap(lidx);
        P.node_level.swap(lev);
        for (int k = 0; k < nb; ++k) P.node_of_bus[P.bus_of_node[k]] = k;
        for (int t = 0; t < ns; ++t) P.level_nodes[t] = t;
    }

    // Y sources per (row bus, col bus): rows of (col, index), sorted by col then index
    std::vector<std::pair<int, int>> yrow;
    auto sources = [&](int i, int j, std::vector<int>& dst) {
        // linear scan of row i (rows are short); keep order of appearance
        int last = -1;
        for (int p = y_row_ptr[i]; p < y_row_ptr[i + 1]; ++p) {
            if (y_col_idx[p] != j) continue;
            if (jac_mode == 0)
                last = p;
            else
                dst.push_back(p);
        }
        if (jac_mode == 0 && last >= 0) dst.push_back(last);
    };
    P.slot_info.assign(static_cast<size_t>(P.n_slots) * 4, 0);
    P.slot_src.clear();
    std::vector<int> slot_a(P.n_slots, -1);
    auto set_slot = [&](int slot, int rb, int cb) {
        int b = static_cast<int>(P.slot_src.size());
        sources(rb, cb, P.slot_src);
        int e = static_cast<int>(P.slot_src.size());
        P.slot_info[4 * slot + 0] = rb;
        P.slot_info[4 * slot + 1] = cb;
        P.slot_info[4 * slot + 2] = b;
        P.slot_info[4 * slot + 3] = e;
    };
    for (int k = 0; k < nb; ++k) set_slot(k, P.bus_of_node[k], P.bus_of_node[k]);
    for (int k = 0; k < nb; ++k)
        for (int p = P.lptr[k]; p < P.lptr[k + 1]; ++p) {
            set_slot(Lbase + p, P.bus_of_node[P.lidx[p]], P.bus_of_node[k]);
            set_slot(Ubase + p, P.bus_of_node[k], P.bus_of_node[P.lidx[p]]);
        }
    // A blocks: diagonal always, off-diagonal where Y has an entry; by block row
    {
        std::vector<std::vector<std::pair<int, int>>> rows(nb);  // (slot, col node)
        for (int k = 0; k < nb; ++k) rows[k].push_back({k, k});
        for (int k = 0; k < nb; ++k)
            for (int p = P.lptr[k]; p < P.lptr[k + 1]; ++p) {
                int a = P.lidx[p];
                int sl = Lbase + p, su = Ubase + p;
                if (P.slot_info[4 * sl + 3] > P.slot_info[4 * sl + 2]) rows[a].push_back({sl, k});
                if (P.slot_info[4 * su + 3] > P.slot_info[4 * su + 2]) rows[k].push_back({su, a});
            }
        P.arow_ptr.assign(nb + 1, 0);
        P.arow.clear();
        int na = 0;
        for (int r = 0; r < nb; ++r) {
            std::sort(rows[r].begin(), rows[r].end(),
                      [](auto const& x, auto const& y) { return x.second < y.second; });
            for (auto const& e : rows[r]) {
                slot_a[e.first] = na;
                P.arow.push_back(na);
                P.arow.push_back(e.second);
                ++na;
            }
            P.arow_ptr[r + 1] = na;
        }
        P.n_a = na;
    }
    P.slot_a = slot_a;
    // the same A blocks by block column (row node), for transposed residuals
    {
        std::vector<int> cnt(nb + 1, 0);
        for (int r = 0; r < nb; ++r)
            for (int e = P.arow_ptr[r]; e < P.arow_ptr[r + 1]; ++e) cnt[P.arow[2 * e + 1] + 1]++;
        for (int c = 0; c < nb; ++c) cnt[c + 1] += cnt[c];
        P.acol_ptr = cnt;
        P.acol.assign(2 * static_cast<size_t>(P.n_a), 0);
        std::vector<int> fp(cnt.begin(), cnt.end() - 1);
        for (int r = 0; r < nb; ++r)
            for (int e = P.arow_ptr[r]; e < P.arow_ptr[r + 1]; ++e) {
                int c = P.arow[2 * e + 1];
                int q = fp[c]++;
                P.acol[2 * q] = P.arow[2 * e];
                P.acol[2 * q + 1] = r;
            }
    }
    // slots that carry Jacobian values, in A order (the fill kernel writes only these)
    P.a_slots.assign(P.n_a, 0);
    for (int sl = 0; sl < P.n_slots; ++sl)
        if (slot_a[sl] >= 0) P.a_slots[slot_a[sl]] = sl;
    P.scale.clear();

    // ---- numeric factorisation schedule (left-looking block Crout) ----
    // Every sparse node m contributes L(a,m) U(m,b) to target (a,b) for all a, b in struct(m).
    // Targets owned by sparse nodes are computed on the level schedule; targets inside the
    // dense tail receive their sparse contributions in one parallel Schur-complement pass
    // (the tail's own contributions are the dense LU's business).
    std::vector<int64_t> cnt(P.n_slots + 1, 0);
    auto target_of = [&](int a, int b) -> int {
        if (a == b) return a;
        if (a < b) {
            int pos = find_in(P.lidx, P.lptr[a], P.lptr[a + 1], b);
            return pos < 0 ? -1 : Ubase + pos;
        }
        int pos = find_in(P.lidx, P.lptr[b], P.lptr[b + 1], a);
        return pos < 0 ? -1 : Lbase + pos;
    };
    for (int m = 0; m < ns; ++m) {
        int b0 = P.lptr[m], e0 = P.lptr[m + 1];
        for (int ia = b0; ia < e0; ++ia)
            for (int ib = b0; ib < e0; ++ib) {
                int t = target_of(P.lidx[ia], P.lidx[ib]);
                if (t < 0) {
                    set_error("symbolic factorisation inconsistent (missing fill slot)");
                    return false;
                }
                cnt[t + 1]++;
            }
    }
    for (int s = 0; s < P.n_slots; ++s) cnt[s + 1] += cnt[s];
    P.n_pairs = cnt[P.n_slots];
    if (P.n_pairs > INT32_MAX / 2) {
        set_error("factorisation schedule too large for 32-bit pair indices");
        return false;
    }
    std::vector<int> spairs(static_cast<size_t>(P.n_pairs) * 2);
    {
        std::vector<int64_t> fp(cnt.begin(), cnt.end() - 1);
        for (int m = 0; m < ns; ++m) {
            int b0 = P.lptr[m], e0 = P.lptr[m + 1];
            for (int ia = b0; ia < e0; ++ia)
                for (int ib = b0; ib < e0; ++ib) {
                    int t = target_of(P.lidx[ia], P.lidx[ib]);
                    int64_t q = fp[t]++;
                    spairs[2 * q] = Lbase + ia;
                    spairs[2 * q + 1] = Ubase + ib;
                }
        }
    }
    auto emit = [&](int s) {
        int pb = static_cast<int>(P.pairs.size() / 2);
        for (int64_t q = cnt[s]; q < cnt[s + 1]; ++q) {
            P.pairs.push_back(spairs[2 * q]);
            P.pairs.push_back(spairs[2 * q + 1]);
        }
        return std::pair<int, int>(pb, static_cast<int>(P.pairs.size() / 2));
    };
    // sparse part: group targets by owner level; phase A holds every slot (D, U row,
    // L column) of the level's nodes, heaviest first; phase B scales the level's L columns
    // by D^-1.
    P.fa_ptr.assign(nlev + 1, 0);
    P.fb_ptr.assign(nlev + 1, 0);
    P.targets.clear();
    P.pairs.clear();
    P.pairs.reserve(spairs.size());
    std::vector<int> lvl_slots;
    for (int h = 0; h < nlev; ++h) {
        lvl_slots.clear();
        for (int t = P.level_ptr[h]; t < P.level_ptr[h + 1]; ++t) {
            int k = P.level_nodes[t];
            lvl_slots.push_back(k);
            for (int p = P.lptr[k]; p < P.lptr[k + 1]; ++p) {
                lvl_slots.push_back(Ubase + p);
                lvl_slots.push_back(Lbase + p);
            }
        }
        std::stable_sort(lvl_slots.begin(), lvl_slots.end(), [&](int x, int y) {
            return (cnt[x + 1] - cnt[x]) > (cnt[y + 1] - cnt[y]);
        });
        for (int s : lvl_slots) {
            auto pe = emit(s);
            // a slot with its Jacobian value and nothing to subtract or invert is final as
            // filled: no target
            if (pe.first == pe.second && s >= nb && slot_a[s] >= 0) continue;
            P.targets.push_back(s);
            P.targets.push_back(pe.first);
            P.targets.push_back(pe.second);
            // bit 0: diagonal (invert); bit 1: the slot holds a Jacobian value (else it
            // starts from zero and is never written by the fill kernel)
            P.targets.push_back((s < nb ? 1 : 0) | (slot_a[s] >= 0 ? 2 : 0));
        }
        P.fa_ptr[h + 1] = static_cast<int>(P.targets.size() / 4);
        for (int t = P.level_ptr[h]; t < P.level_ptr[h + 1]; ++t) {
            int k = P.level_nodes[t];
            for (int p = P.lptr[k]; p < P.lptr[k + 1]; ++p) {
                P.scale.push_back(Lbase + p);
                P.scale.push_back(k);
            }
        }
        P.fb_ptr[h + 1] = static_cast<int>(P.scale.size() / 2);
    }
    // dense tail: (slot, pair_begin, pair_end, dense block position r*T + c)
    // every one of the T^2 tail blocks gets a target, so the gather overwrites the whole
    // dense block each iteration; blocks outside the symbolic structure (an extended tail is
    // not full) have no pairs and no Jacobian value and are written as zero.  Targets are in
    // row-major block order: consecutive threads of one scenario write adjacent blocks.
    P.schur.assign(static_cast<size_t>(T) * T * 4, 0);
    {
        auto hs = [&](int sl) { return slot_a[sl] >= 0 ? (1 << 30) : 0; };
        auto put = [&](int r, int c, int slot, bool has) {
            const size_t q = (static_cast<size_t>(r) * T + c) * 4;
            if (has) {
                auto pe = emit(slot);
                P.schur[q] = slot;
                P.schur[q + 1] = pe.first;
                P.schur[q + 2] = pe.second;
                P.schur[q + 3] = (r * T + c) | hs(slot);
            } else {
                const int pz = static_cast<int>(P.pairs.size() / 2);
                P.schur[q] = ns + r;
                P.schur[q + 1] = pz;
                P.schur[q + 2] = pz;
                P.schur[q + 3] = r * T + c;
            }
        };
        std::vector<int> ucol(T);
        for (int r = 0; r < T; ++r) {
            const int kr = ns + r;
            // U(kr, a) for a > kr and L(a, kr): positions of row kr's column structure
            std::fill(ucol.begin(), ucol.end(), -1);
            for (int p = P.lptr[kr]; p < P.lptr[kr + 1]; ++p) ucol[P.lidx[p] - ns] = p;
            for (int c = 0; c < T; ++c) {
                if (c == r) {
                    put(r, c, kr, true);
                } else if (c > r) {
                    const int p = ucol[c];
                    put(r, c, p >= 0 ? Ubase + p : -1, p >= 0);
                } else {
                    // L(kr, ns + c) lives in column ns + c's structure
                    const int kc = ns + c;
                    const int p = find_in(P.lidx, P.lptr[kc], P.lptr[kc + 1], kr);
                    put(r, c, p >= 0 ? Lbase + p : -1, p >= 0);
                }
            }
        }
    }

    // ---- forward-solve row lists (sparse columns only; the tail's own columns are in the
    // dense factor) ----
    P.rptr.assign(nb + 1, 0);
    for (int m = 0; m < ns; ++m)
        for (int p = P.lptr[m]; p < P.lptr[m + 1]; ++p) P.rptr[P.lidx[p] + 1]++;
    for (int k = 0; k < nb; ++k) P.rptr[k + 1] += P.rptr[k];
    P.rlist.assign(static_cast<size_t>(P.rptr[nb]) * 2, 0);
    {
        std::vector<int> fp(P.rptr.begin(), P.rptr.end() - 1);
        for (int m = 0; m < ns; ++m)
            for (int p = P.lptr[m]; p < P.lptr[m + 1]; ++p) {
                int k = P.lidx[p];
                int q = fp[k]++;
                P.rlist[2 * q] = Lbase + p;
                P.rlist[2 * q + 1] = m;
            }
    }

    // ---- reference variable / equation order ----
    std::vector<int> ang(n_bus, -1), mag(n_bus, -1), peq(n_bus, -1), qeq(n_bus, -1);
    {
        int c = 0;
        for (int i = 0; i < n_bus; ++i)
            if (bus_type[i] != 2) ang[i] = c++;
        for (int i = 0; i < n_bus; ++i)
            if (bus_type[i] == 0) mag[i] = c++;
        int r = 0;
        for (int i = 0; i < n_bus; ++i) {
            if (bus_type[i] == 2) continue;
            peq[i] = r++;
            if (bus_type[i] == 0) qeq[i] = r++;
        }
    }
    P.var_of_comp.assign(2 * nb, -1);
    P.eq_of_comp.assign(2 * nb, -1);
    for (int k = 0; k < nb; ++k) {
        int i = P.bus_of_node[k];
        P.var_of_comp[2 * k] = ang[i];
        P.var_of_comp[2 * k + 1] = mag[i];
        P.eq_of_comp[2 * k] = peq[i];
        P.eq_of_comp[2 * k + 1] = qeq[i];
    }
    return true;
}

}  // namespace gapk

namespace gapk {

// Row permutation giving a zero-free diagonal (maximum transversal by depth-first augmenting
// paths, Duff's MC21 method): on success rp[i] is the original row placed at position i, with
// A[rp[i]][i] structurally non-zero.  Returns false when the pattern is structurally singular.
static bool zero_free_diagonal(int n, const int* row_ptr, const int* col_idx,
                               std::vector<int>& rp) {
    std::vector<int> col_row(n, -1), row_col(n, -1), seen(n, -1);
    std::vector<int> rows, pos, via;
    for (int r0 = 0; r0 < n; ++r0) {
        int found = -1;
        for (int p = row_ptr[r0]; p < row_ptr[r0 + 1]; ++p)
            if (col_row[col_idx[p]] < 0) {
                found = col_idx[p];
                break;
            }
        rows.assign(1, r0);
        pos.assign(1, row_ptr[r0]);
        via.clear();
        // depth-first search for an augmenting path; via[d] leads from rows[d] to rows[d+1]
        while (found < 0 && !rows.empty()) {
            const int d = static_cast<int>(rows.size()) - 1;
            const int u = rows[d];
            if (pos[d] == row_ptr[u + 1]) {
                rows.pop_back();
                pos.pop_back();
                if (!via.empty()) via.pop_back();
                continue;
            }
            const int c = col_idx[pos[d]++];
            if (seen[c] == r0) continue;
            seen[c] = r0;
            if (col_row[c] < 0) {
                found = c;
                break;
            }
            via.push_back(c);
            rows.push_back(col_row[c]);
            pos.push_back(row_ptr[col_row[c]]);
        }
        if (found < 0) return false;
        int c = found;
        for (int d = static_cast<int>(rows.size()) - 1; d >= 0; --d) {
            col_row[c] = rows[d];
            row_col[rows[d]] = c;
            c = d > 0 ? via[d - 1] : -1;
        }
    }
    rp = col_row;
    return true;
}

bool analyze_general(int n, int nnz, const int* row_ptr, const int* col_idx, int dense_min,
                     NRPlanHost& P, std::vector<int>& rp, std::vector<int>& val_map) {
    if (n <= 0 || nnz <= 0 || row_ptr[0] != 0 || row_ptr[n] != nnz) {
        set_error("matrix must be square with a consistent, non-empty CSR pattern");
        return false;
    }
    for (int i = 0; i < n; ++i)
        if (row_ptr[i + 1] < row_ptr[i]) {
            set_error("row_ptr not monotone");
            return false;
        }
    for (int p = 0; p < nnz; ++p)
        if (col_idx[p] < 0 || col_idx[p] >= n) {
            set_error("col_idx out of range");
            return false;
        }
    if (!zero_free_diagonal(n, row_ptr, col_idx, rp)) {
        set_error("matrix is structurally singular (no zero-free diagonal)");
        return false;
    }
    // B = P A: row i of B is row rp[i] of A; val_map[e] = index in A of B's entry e
    std::vector<int> brp(n + 1, 0), bci;
    bci.reserve(nnz);
    val_map.clear();
    val_map.reserve(nnz);
    for (int i = 0; i < n; ++i) {
        int r = rp[i];
        for (int p = row_ptr[r]; p < row_ptr[r + 1]; ++p) {
            bci.push_back(col_idx[p]);
            val_map.push_back(p);
        }
        brp[i + 1] = static_cast<int>(bci.size());
    }
    std::vector<int> bt(n, 0);  // every position is an unknown ("PQ")
    if (!analyze_nr(n, nnz, brp.data(), bci.data(), bt.data(), 1, 0, dense_min, P)) return false;
    return true;
}

}  // namespace gapk
