// Host construction of the device sweep schedule (see schedule.h).
#include "schedule.h"
#include "cluster_schedule.h"

#include <algorithm>
#include <cstring>
#include <cmath>
#include <numeric>
#include <queue>
#include <tuple>

namespace swb {
namespace {

struct Constraint {
    uint32_t n[4];
    int count;          // 2 or 4
    uint32_t def_index;
};

// Recursive coordinate bisection into `parts` balanced parts, choosing on
// every split the axis and the cut position (within the balance tolerance)
// that cut the fewest constraints.  Items are groups of nodes that must
// stay together; constraints are given over items.
class Bisector {
public:
    Bisector(const std::vector<std::array<double, 3>>& item_pos,
             const std::vector<double>& item_weight,
             const std::vector<std::vector<uint32_t>>& cons_items,
             double tolerance)
        : pos_(item_pos), weight_(item_weight), cons_(cons_items),
          tol_(tolerance), part_(item_pos.size(), 0), rank_(item_pos.size(), 0) {}

    std::vector<int> run(int parts) {
        std::vector<uint32_t> items(pos_.size());
        std::iota(items.begin(), items.end(), 0u);
        std::vector<uint32_t> cons;
        for (uint32_t c = 0; c < cons_.size(); ++c) cons.push_back(c);
        split(items, cons, parts, 0);
        return part_;
    }

private:
    void split(std::vector<uint32_t>& items, std::vector<uint32_t>& cons,
               int parts, int base) {
        if (parts <= 1 || items.size() <= 1) {
            for (uint32_t i : items) part_[i] = base;
            return;
        }
        const int left_parts = parts / 2;
        double total = 0.0;
        for (uint32_t i : items) total += weight_[i];
        const double target = total * left_parts / parts;
        const size_t n = items.size();
        double best_score = 1e300;
        int best_axis = 0;
        size_t best_index = n / 2;
        std::vector<uint32_t> sorted(items);
        std::vector<int64_t> diff(n + 2);
        std::vector<double> prefix(n + 1);
        for (int axis = 0; axis < 3; ++axis) {
            std::stable_sort(sorted.begin(), sorted.end(), [&](uint32_t l, uint32_t r) {
                if (pos_[l][axis] != pos_[r][axis]) return pos_[l][axis] < pos_[r][axis];
                return l < r;
            });
            for (size_t k = 0; k < n; ++k) rank_[sorted[k]] = static_cast<uint32_t>(k);
            prefix[0] = 0.0;
            for (size_t k = 0; k < n; ++k) prefix[k + 1] = prefix[k] + weight_[sorted[k]];
            std::fill(diff.begin(), diff.end(), 0);
            for (uint32_t c : cons) {
                uint32_t lo = UINT32_MAX, hi = 0;
                for (uint32_t it : cons_[c]) {
                    lo = std::min(lo, rank_[it]);
                    hi = std::max(hi, rank_[it]);
                }
                if (lo == hi) continue;
                diff[lo + 1] += 1;
                diff[hi + 1] -= 1;
            }
            int64_t cut = 0;
            size_t closest = 1;
            for (size_t i = 1; i < n; ++i)
                if (std::fabs(prefix[i] - target) < std::fabs(prefix[closest] - target))
                    closest = i;
            for (size_t i = 1; i < n; ++i) {
                cut += diff[i];
                const double imbalance = std::fabs(prefix[i] - target) / total;
                if (imbalance > tol_ && i != closest) continue;
                const double score = static_cast<double>(cut) + 4.0 * imbalance * cons.size();
                if (score < best_score) {
                    best_score = score;
                    best_axis = axis;
                    best_index = i;
                }
            }
        }
        std::vector<uint32_t> best_sorted(items);
        std::stable_sort(best_sorted.begin(), best_sorted.end(), [&](uint32_t l, uint32_t r) {
            if (pos_[l][best_axis] != pos_[r][best_axis])
                return pos_[l][best_axis] < pos_[r][best_axis];
            return l < r;
        });
        for (size_t k = 0; k < n; ++k) rank_[best_sorted[k]] = static_cast<uint32_t>(k);
        std::vector<uint32_t> left(best_sorted.begin(), best_sorted.begin() + best_index);
        std::vector<uint32_t> right(best_sorted.begin() + best_index, best_sorted.end());
        std::vector<uint32_t> lc, rc;
        for (uint32_t c : cons) {
            bool all_left = true, all_right = true;
            for (uint32_t it : cons_[c]) {
                if (rank_[it] < best_index) all_right = false;
                else all_left = false;
            }
            if (all_left) lc.push_back(c);
            else if (all_right) rc.push_back(c);
        }
        items.clear();
        items.shrink_to_fit();
        cons.clear();
        cons.shrink_to_fit();
        split(left, lc, left_parts, base);
        split(right, rc, parts - left_parts, base + left_parts);
    }

    const std::vector<std::array<double, 3>>& pos_;
    const std::vector<double>& weight_;
    const std::vector<std::vector<uint32_t>>& cons_;
    double tol_;
    std::vector<int> part_;
    std::vector<uint32_t> rank_;
};

// DSatur colouring of constraints that conflict when they share a node.
// Returns colour per constraint and the colour count.
int dsatur(const std::vector<const Constraint*>& cons, std::vector<int>& colour) {
    const size_t m = cons.size();
    colour.assign(m, -1);
    if (m == 0) return 0;
    // node -> constraints
    std::vector<uint32_t> nodes;
    for (const Constraint* c : cons)
        for (int k = 0; k < c->count; ++k) nodes.push_back(c->n[k]);
    std::sort(nodes.begin(), nodes.end());
    nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
    auto node_id = [&](uint32_t n) {
        return static_cast<size_t>(std::lower_bound(nodes.begin(), nodes.end(), n) - nodes.begin());
    };
    std::vector<uint32_t> off(nodes.size() + 1, 0);
    std::vector<std::array<uint32_t, 4>> cn(m);
    for (size_t i = 0; i < m; ++i)
        for (int k = 0; k < cons[i]->count; ++k) {
            cn[i][k] = static_cast<uint32_t>(node_id(cons[i]->n[k]));
            ++off[cn[i][k] + 1];
        }
    for (size_t v = 0; v < nodes.size(); ++v) off[v + 1] += off[v];
    std::vector<uint32_t> inc(off.back());
    std::vector<uint32_t> cur(off.begin(), off.end() - 1);
    for (size_t i = 0; i < m; ++i)
        for (int k = 0; k < cons[i]->count; ++k) inc[cur[cn[i][k]]++] = static_cast<uint32_t>(i);
    std::vector<uint32_t> degree(m, 0);
    for (size_t i = 0; i < m; ++i)
        for (int k = 0; k < cons[i]->count; ++k) degree[i] += off[cn[i][k] + 1] - off[cn[i][k]] - 1;
    std::vector<std::vector<uint64_t>> used(m);
    std::vector<uint32_t> sat(m, 0);
    using Key = std::tuple<uint32_t, uint32_t, int64_t>;  // sat, degree, -index
    std::priority_queue<Key> heap;
    for (size_t i = 0; i < m; ++i) heap.emplace(0u, degree[i], -static_cast<int64_t>(i));
    int colours = 0;
    auto has = [&](size_t i, int c) {
        const auto& u = used[i];
        return static_cast<size_t>(c / 64) < u.size() && ((u[c / 64] >> (c % 64)) & 1u);
    };
    while (!heap.empty()) {
        auto [s, dg, ni] = heap.top();
        heap.pop();
        const size_t i = static_cast<size_t>(-ni);
        if (colour[i] >= 0 || s != sat[i]) continue;
        int c = 0;
        while (has(i, c)) ++c;
        colour[i] = c;
        colours = std::max(colours, c + 1);
        for (int k = 0; k < cons[i]->count; ++k) {
            const uint32_t v = cn[i][k];
            for (uint32_t q = off[v]; q < off[v + 1]; ++q) {
                const uint32_t j = inc[q];
                if (colour[j] >= 0 || has(j, c)) continue;
                auto& u = used[j];
                if (u.size() <= static_cast<size_t>(c / 64)) u.resize(c / 64 + 1, 0);
                u[c / 64] |= uint64_t{1} << (c % 64);
                ++sat[j];
                heap.emplace(sat[j], degree[j], -static_cast<int64_t>(j));
            }
        }
    }
    return colours;
}

}  // namespace

// Node partition into `parts` by cut-minimising recursive coordinate
// bisection; `grouped_nodes` form one item that is never split.  Item
// weight = 1 + half the number of constraint incidences (work proxy).
std::vector<int> bisect_nodes(const OwnedDefinition& d, const std::vector<uint32_t>& grouped_nodes, int parts,
                              double tolerance) {
    const uint32_t N = static_cast<uint32_t>(d.nodes.size());
    std::vector<uint32_t> incidence(N, 0);
    for (const auto& c : d.constraints) {
        ++incidence[c.first_node];
        ++incidence[c.second_node];
    }
    for (const auto& h : d.dihedrals)
        for (uint64_t n : h.nodes) ++incidence[n];
    std::vector<uint32_t> item_of(N);
    std::vector<std::array<double, 3>> ipos;
    std::vector<double> iweight;
    std::vector<uint8_t> grouped(N, 0);
    for (uint32_t n : grouped_nodes) grouped[n] = 1;
    int32_t group = -1;
    std::array<double, 3> gsum{0, 0, 0};
    double gw = 0.0;
    uint32_t gcount = 0;
    for (uint32_t n = 0; n < N; ++n) {
        const auto& p = d.nodes[n].position;
        const double w = 1.0 + 0.5 * incidence[n];
        if (grouped[n]) {
            if (group < 0) {
                group = static_cast<int32_t>(ipos.size());
                ipos.push_back({0, 0, 0});
                iweight.push_back(0);
            }
            item_of[n] = static_cast<uint32_t>(group);
            gsum[0] += p.x; gsum[1] += p.y; gsum[2] += p.z;
            gw += w;
            ++gcount;
        } else {
            item_of[n] = static_cast<uint32_t>(ipos.size());
            ipos.push_back({p.x, p.y, p.z});
            iweight.push_back(w);
        }
    }
    if (group >= 0) {
        ipos[group] = {gsum[0] / gcount, gsum[1] / gcount, gsum[2] / gcount};
        iweight[group] = gw;
    }
    std::vector<std::vector<uint32_t>> cons_items;
    cons_items.reserve(d.constraints.size() + d.dihedrals.size());
    for (const auto& c : d.constraints)
        cons_items.push_back({item_of[c.first_node], item_of[c.second_node]});
    for (const auto& h : d.dihedrals)
        cons_items.push_back({item_of[h.nodes[0]], item_of[h.nodes[1]], item_of[h.nodes[2]], item_of[h.nodes[3]]});
    const std::vector<int> item_part = Bisector(ipos, iweight, cons_items, tolerance).run(parts);
    std::vector<int> part(N);
    for (uint32_t n = 0; n < N; ++n) part[n] = item_part[item_of[n]];
    return part;
}

int dsatur_colour(const std::vector<std::array<uint32_t, 4>>& nodes, const std::vector<int>& counts,
                  std::vector<int>& colour) {
    std::vector<Constraint> cons(nodes.size());
    std::vector<const Constraint*> ptrs(nodes.size());
    for (size_t i = 0; i < nodes.size(); ++i) {
        cons[i] = {{nodes[i][0], nodes[i][1], nodes[i][2], nodes[i][3]}, counts[i], static_cast<uint32_t>(i)};
        ptrs[i] = &cons[i];
    }
    return dsatur(ptrs, colour);
}

Schedule build_schedule(const OwnedDefinition& d,
                        const std::vector<uint32_t>& suspension_nodes,
                        const ScheduleOptions& opt) {
    Schedule S;
    const uint32_t N = static_cast<uint32_t>(d.nodes.size());
    const int G = std::max(1, opt.blocks);
    S.blocks = G;
    S.node_count = N;
    const int L = opt.global_only ? 0 : std::clamp(opt.levels, 1, kMaxLevels);

    // Constraints of both kinds.
    std::array<std::vector<Constraint>, kKinds> all;
    for (uint32_t i = 0; i < d.constraints.size(); ++i) {
        const auto& c = d.constraints[i];
        all[0].push_back({{static_cast<uint32_t>(c.first_node),
                           static_cast<uint32_t>(c.second_node), 0, 0}, 2, i});
    }
    for (uint32_t i = 0; i < d.dihedrals.size(); ++i) {
        const auto& h = d.dihedrals[i];
        all[1].push_back({{static_cast<uint32_t>(h.nodes[0]), static_cast<uint32_t>(h.nodes[1]),
                           static_cast<uint32_t>(h.nodes[2]), static_cast<uint32_t>(h.nodes[3])},
                          4, i});
    }

    // ---- level 1: node partition (suspension nodes grouped) ---------------
    const std::vector<int> part1 = bisect_nodes(d, suspension_nodes, G, opt.balance_tolerance);

    // Slots: level-1 part-major, node index within.
    S.l1_begin.assign(G + 1, 0);
    for (uint32_t n = 0; n < N; ++n) ++S.l1_begin[part1[n] + 1];
    for (int b = 0; b < G; ++b) S.l1_begin[b + 1] += S.l1_begin[b];
    S.node_of_slot.assign(N, 0);
    S.slot_of_node.assign(N, 0);
    {
        std::vector<uint32_t> cur(S.l1_begin.begin(), S.l1_begin.end() - 1);
        for (uint32_t n = 0; n < N; ++n) {
            const uint32_t s = cur[part1[n]]++;
            S.node_of_slot[s] = n;
            S.slot_of_node[n] = s;
        }
    }
    for (int b = 0; b < G; ++b)
        S.max_patch_nodes = std::max<int>(S.max_patch_nodes, S.l1_begin[b + 1] - S.l1_begin[b]);
    if (S.max_patch_nodes > 65535)
        raise(SWB_UNSUPPORTED, "a level-1 patch exceeds 65535 nodes; use more blocks");
    if (!suspension_nodes.empty()) S.suspension_block = part1[suspension_nodes[0]];

    // ---- levels: assign interior constraints, repartition the rest --------
    std::array<std::vector<const Constraint*>, kKinds> remaining;
    for (int k = 0; k < kKinds; ++k)
        for (const Constraint& c : all[k]) remaining[k].push_back(&c);

    // per-level per-kind per-block constraint lists
    std::vector<std::array<std::vector<std::vector<const Constraint*>>, kKinds>> lists(kMaxLevels);
    std::vector<std::vector<int>> level_part(kMaxLevels);  // node -> part (or -1)
    int used_levels = 0;
    for (int level = 0; level < L; ++level) {
        std::vector<int> part(N, -1);
        if (level == 0) {
            part = part1;
        } else {
            // items = nodes touched by remaining constraints
            std::vector<int32_t> item(N, -1);
            std::vector<std::array<double, 3>> p2;
            std::vector<double> w2;
            std::vector<uint32_t> node_of_item;
            for (int k = 0; k < kKinds; ++k)
                for (const Constraint* c : remaining[k])
                    for (int q = 0; q < c->count; ++q) {
                        const uint32_t n = c->n[q];
                        if (item[n] < 0) {
                            item[n] = static_cast<int32_t>(p2.size());
                            const auto& pp = d.nodes[n].position;
                            p2.push_back({pp.x, pp.y, pp.z});
                            w2.push_back(0.0);
                            node_of_item.push_back(n);
                        }
                        w2[item[n]] += 1.0;
                    }
            if (p2.empty()) break;
            std::vector<std::vector<uint32_t>> ci;
            for (int k = 0; k < kKinds; ++k)
                for (const Constraint* c : remaining[k]) {
                    std::vector<uint32_t> it;
                    for (int q = 0; q < c->count; ++q) it.push_back(static_cast<uint32_t>(item[c->n[q]]));
                    ci.push_back(std::move(it));
                }
            std::vector<int> ip = Bisector(p2, w2, ci, opt.balance_tolerance).run(G);
            for (size_t i = 0; i < ip.size(); ++i) part[node_of_item[i]] = ip[i];
        }
        level_part[level] = part;
        bool any = false;
        for (int k = 0; k < kKinds; ++k) {
            lists[level][k].assign(G, {});
            std::vector<const Constraint*> rest;
            for (const Constraint* c : remaining[k]) {
                const int p0 = part[c->n[0]];
                bool inside = p0 >= 0;
                for (int q = 1; q < c->count && inside; ++q) inside = part[c->n[q]] == p0;
                if (inside) {
                    lists[level][k][p0].push_back(c);
                    any = true;
                } else {
                    rest.push_back(c);
                }
            }
            remaining[k].swap(rest);
        }
        if (!any && level > 0) break;
        used_levels = level + 1;
    }
    S.levels = used_levels;

    // ---- per level tables ---------------------------------------------------
    std::vector<uint8_t> touched_outside_l1(N, 0);
    for (int level = 0; level < used_levels; ++level) {
        // Patch node lists for levels >= 2: nodes referenced by that level.
        std::vector<int32_t> local(N, -1);
        if (level > 0) {
            S.patch_begin[level].assign(G + 1, 0);
            for (int b = 0; b < G; ++b) {
                std::vector<uint32_t> nodes;
                for (int k = 0; k < kKinds; ++k)
                    for (const Constraint* c : lists[level][k][b])
                        for (int q = 0; q < c->count; ++q) nodes.push_back(c->n[q]);
                std::sort(nodes.begin(), nodes.end(), [&](uint32_t x, uint32_t y) {
                    return S.slot_of_node[x] < S.slot_of_node[y];
                });
                nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
                if (nodes.size() > 65535)
                    raise(SWB_UNSUPPORTED, "a gathered patch exceeds 65535 nodes");
                for (size_t i = 0; i < nodes.size(); ++i) {
                    local[nodes[i]] = static_cast<int32_t>(i);
                    S.patch_slots[level].push_back(S.slot_of_node[nodes[i]]);
                    touched_outside_l1[nodes[i]] = 1;
                }
                S.patch_begin[level][b + 1] = S.patch_begin[level][b] + static_cast<uint32_t>(nodes.size());
                S.max_gather_nodes = std::max<int>(S.max_gather_nodes, static_cast<int>(nodes.size()));
            }
        }
        for (int k = 0; k < kKinds; ++k) {
            Table& T = S.tables[level][k];
            T.block_begin.assign(G + 1, 0);
            std::vector<std::vector<const Constraint*>> staged(G);
            std::vector<std::vector<uint32_t>> stage_sizes(G);
            int max_stages = 0;
            for (int b = 0; b < G; ++b) {
                const auto& cl = lists[level][k][b];
                std::vector<int> colour;
                const int colours = dsatur(cl, colour);
                max_stages = std::max(max_stages, colours);
                std::vector<uint32_t> count(colours, 0);
                for (int c : colour) ++count[c];
                // stable colour-major order
                std::vector<uint32_t> idx(cl.size());
                std::iota(idx.begin(), idx.end(), 0u);
                std::stable_sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) {
                    return colour[x] < colour[y];
                });
                for (uint32_t i : idx) staged[b].push_back(cl[i]);
                stage_sizes[b] = count;
            }
            T.stages = max_stages;
            T.stage_offsets.assign(static_cast<size_t>(G) * (max_stages + 1), 0);
            for (int b = 0; b < G; ++b) {
                const uint32_t count = static_cast<uint32_t>(staged[b].size());
                const uint32_t padded = (count + 3u) & ~3u;
                T.block_begin[b + 1] = T.block_begin[b] + padded;
                T.max_block_count = std::max(T.max_block_count, padded);
                uint32_t off = 0;
                for (int s = 0; s < max_stages; ++s) {
                    T.stage_offsets[static_cast<size_t>(b) * (max_stages + 1) + s] = off;
                    if (s < static_cast<int>(stage_sizes[b].size())) off += stage_sizes[b][s];
                }
                T.stage_offsets[static_cast<size_t>(b) * (max_stages + 1) + max_stages] = off;
                const uint32_t base = (level == 0) ? S.l1_begin[b] : 0;
                for (uint32_t i = 0; i < padded; ++i) {
                    if (i < count) {
                        const Constraint* c = staged[b][i];
                        uint32_t li[4] = {0, 0, 0, 0};
                        for (int q = 0; q < c->count; ++q)
                            li[q] = level == 0 ? S.slot_of_node[c->n[q]] - base
                                               : static_cast<uint32_t>(local[c->n[q]]);
                        T.ab.push_back(li[0] | (li[1] << 16));
                        if (k == 1) T.cd.push_back(li[2] | (li[3] << 16));
                        if (k == 0) {
                            const auto& dc = d.constraints[c->def_index];
                            const bool stitch = dc.kind == SWB_CONSTRAINT_SEAM_STITCH;
                            T.rest.push_back(stitch ? 0.0f : static_cast<float>(dc.rest_length));
                            float cp = stitch ? 0.0f : static_cast<float>(dc.compliance);
                            if (dc.kind == SWB_CONSTRAINT_CABLE) cp = std::copysign(std::fabs(cp), -1.0f);
                            T.comp.push_back(cp);
                        } else {
                            const auto& dh = d.dihedrals[c->def_index];
                            T.rest.push_back(static_cast<float>(dh.rest_angle));
                            T.comp.push_back(static_cast<float>(dh.compliance));
                        }
                        T.def_index.push_back(c->def_index);
                        T.valid.push_back(1);
                    } else {
                        T.ab.push_back(0);
                        if (k == 1) T.cd.push_back(0);
                        T.rest.push_back(0.0f);
                        T.comp.push_back(0.0f);
                        T.def_index.push_back(0);
                        T.valid.push_back(0);
                    }
                }
                S.level_constraints[level] += count;
            }
        }
    }

    // ---- global leftovers -------------------------------------------------
    for (int k = 0; k < kKinds; ++k) {
        GlobalTable& T = S.global[k];
        std::vector<int> colour;
        const int colours = dsatur(remaining[k], colour);
        std::vector<uint32_t> idx(remaining[k].size());
        std::iota(idx.begin(), idx.end(), 0u);
        std::stable_sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) {
            return colour[x] < colour[y];
        });
        T.colour_offsets.assign(colours + 1, 0);
        for (int c : colour) ++T.colour_offsets[c + 1];
        for (int c = 0; c < colours; ++c) T.colour_offsets[c + 1] += T.colour_offsets[c];
        for (uint32_t i : idx) {
            const Constraint* c = remaining[k][i];
            T.a.push_back(S.slot_of_node[c->n[0]]);
            T.b.push_back(S.slot_of_node[c->n[1]]);
            for (int q = 0; q < c->count; ++q) touched_outside_l1[c->n[q]] = 1;
            if (k == 1) {
                T.c.push_back(S.slot_of_node[c->n[2]]);
                T.d.push_back(S.slot_of_node[c->n[3]]);
                const auto& dh = d.dihedrals[c->def_index];
                T.rest.push_back(static_cast<float>(dh.rest_angle));
                T.comp.push_back(static_cast<float>(dh.compliance));
            } else {
                const auto& dc = d.constraints[c->def_index];
                const bool stitch = dc.kind == SWB_CONSTRAINT_SEAM_STITCH;
                T.rest.push_back(stitch ? 0.0f : static_cast<float>(dc.rest_length));
                float cp = stitch ? 0.0f : static_cast<float>(dc.compliance);
                if (dc.kind == SWB_CONSTRAINT_CABLE) cp = std::copysign(std::fabs(cp), -1.0f);
                T.comp.push_back(cp);
            }
            T.def_index.push_back(c->def_index);
        }
        S.global_constraints += remaining[k].size();
    }

    // ---- sweep orders --------------------------------------------------------
    for (int k = 0; k < kKinds; ++k) {
        auto& order = k == 0 ? S.distance_order : S.dihedral_order;
        for (int level = 0; level < used_levels; ++level) {
            const Table& T = S.tables[level][k];
            for (size_t i = 0; i < T.def_index.size(); ++i)
                if (T.valid[i]) order.push_back(T.def_index[i]);
        }
        for (uint32_t i : S.global[k].def_index) order.push_back(i);
    }

    // ---- seam closing pass: level scheduling in sweep order -------------------
    {
        std::vector<int32_t> node_stage(N, -1);
        std::vector<std::pair<int, uint64_t>> st;
        for (uint64_t i : S.distance_order) {
            const auto& c = d.constraints[i];
            if (c.kind != SWB_CONSTRAINT_SEAM_STITCH) continue;
            const int s = std::max(node_stage[c.first_node], node_stage[c.second_node]) + 1;
            node_stage[c.first_node] = node_stage[c.second_node] = s;
            st.emplace_back(s, i);
            touched_outside_l1[c.first_node] = touched_outside_l1[c.second_node] = 1;
        }
        std::stable_sort(st.begin(), st.end(),
                         [](const auto& x, const auto& y) { return x.first < y.first; });
        int stages = st.empty() ? 0 : st.back().first + 1;
        S.seam_stage_offsets.assign(stages + 1, 0);
        for (const auto& [s, i] : st) {
            ++S.seam_stage_offsets[s + 1];
            S.seam_a.push_back(S.slot_of_node[d.constraints[i].first_node]);
            S.seam_b.push_back(S.slot_of_node[d.constraints[i].second_node]);
        }
        for (int s = 0; s < stages; ++s) S.seam_stage_offsets[s + 1] += S.seam_stage_offsets[s];
    }

    // ---- level-1 interface -----------------------------------------------------
    S.iface_begin.assign(G + 1, 0);
    for (int b = 0; b < G; ++b) {
        for (uint32_t s = S.l1_begin[b]; s < S.l1_begin[b + 1]; ++s)
            if (touched_outside_l1[S.node_of_slot[s]])
                S.iface_local.push_back(static_cast<uint16_t>(s - S.l1_begin[b]));
        S.iface_begin[b + 1] = static_cast<uint32_t>(S.iface_local.size());
    }
    return S;
}

}  // namespace swb

namespace swb {

std::vector<uint32_t> suspension_endpoint_nodes(const OwnedDefinition& d) {
    std::vector<uint32_t> nodes;
    if (!d.has_suspension) return nodes;
    for (const auto& g : d.segments)
        for (const swb_suspension_endpoint* e : {&g.from, &g.to}) {
            if (e->kind == SWB_ENDPOINT_SURFACE_ATTACHMENT) {
                for (const auto& a : d.attachments)
                    if (a.stable_id == e->stable_id) nodes.push_back(static_cast<uint32_t>(a.node));
            } else if (e->kind == SWB_ENDPOINT_JUNCTION) {
                for (const auto& j : d.junctions)
                    if (j.stable_id == e->stable_id) nodes.push_back(static_cast<uint32_t>(j.node));
            }
        }
    std::sort(nodes.begin(), nodes.end());
    nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
    return nodes;
}

void verify_schedule(const OwnedDefinition& d, const std::vector<uint32_t>& suspension_nodes,
                     const Schedule& S) {
    auto fail = [](const std::string& what) { raise(SWB_INVALID_ARGUMENT, "schedule invariant: " + what); };
    const uint32_t N = static_cast<uint32_t>(d.nodes.size());
    const int G = S.blocks;
    // slots
    if (S.node_of_slot.size() != N || S.slot_of_node.size() != N) fail("slot map size");
    for (uint32_t n = 0; n < N; ++n)
        if (S.node_of_slot[S.slot_of_node[n]] != n) fail("slot map is not a bijection");
    if (S.l1_begin.size() != static_cast<size_t>(G) + 1 || S.l1_begin[0] != 0 || S.l1_begin[G] != N)
        fail("level-1 ranges");
    std::vector<int> l1_block(N, -1);
    for (int b = 0; b < G; ++b)
        for (uint32_t s = S.l1_begin[b]; s < S.l1_begin[b + 1]; ++s) l1_block[S.node_of_slot[s]] = b;
    for (uint32_t n : suspension_nodes)
        if (l1_block[n] != S.suspension_block) fail("suspension node outside the owner patch");
    std::array<std::vector<uint32_t>, kKinds> seen;
    seen[0].assign(d.constraints.size(), 0);
    seen[1].assign(d.dihedrals.size(), 0);
    std::vector<uint8_t> outside(N, 0);
    std::vector<int64_t> stamp(N, -1);
    int64_t epoch = 0;
    auto nodes_of = [&](int k, uint32_t i, uint32_t out[4]) {
        if (k == 0) {
            out[0] = static_cast<uint32_t>(d.constraints[i].first_node);
            out[1] = static_cast<uint32_t>(d.constraints[i].second_node);
            return 2;
        }
        for (int q = 0; q < 4; ++q) out[q] = static_cast<uint32_t>(d.dihedrals[i].nodes[q]);
        return 4;
    };
    for (int level = 0; level < S.levels; ++level) {
        // patch membership for this level
        std::vector<int> owner(N, -1);
        std::vector<std::vector<uint32_t>> local_to_node(G);
        if (level == 0) {
            owner = l1_block;
            for (int b = 0; b < G; ++b)
                for (uint32_t s = S.l1_begin[b]; s < S.l1_begin[b + 1]; ++s)
                    local_to_node[b].push_back(S.node_of_slot[s]);
        } else {
            for (int b = 0; b < G; ++b)
                for (uint32_t i = S.patch_begin[level][b]; i < S.patch_begin[level][b + 1]; ++i) {
                    const uint32_t n = S.node_of_slot[S.patch_slots[level][i]];
                    if (owner[n] >= 0) fail("gathered patches overlap");
                    owner[n] = b;
                    local_to_node[b].push_back(n);
                }
        }
        for (int k = 0; k < kKinds; ++k) {
            const Table& T = S.tables[level][k];
            for (int b = 0; b < G; ++b) {
                const uint32_t bb = T.block_begin[b];
                for (int s = 0; s < T.stages; ++s) {
                    ++epoch;
                    const size_t o = static_cast<size_t>(b) * (T.stages + 1) + s;
                    for (uint32_t i = T.stage_offsets[o]; i < T.stage_offsets[o + 1]; ++i) {
                        const uint32_t e = bb + i;
                        if (!T.valid[e]) fail("padding inside a stage");
                        uint32_t li[4] = {T.ab[e] & 0xffffu, T.ab[e] >> 16, 0, 0};
                        if (k == 1) { li[2] = T.cd[e] & 0xffffu; li[3] = T.cd[e] >> 16; }
                        uint32_t dn[4];
                        const int cnt = nodes_of(k, T.def_index[e], dn);
                        ++seen[k][T.def_index[e]];
                        for (int q = 0; q < cnt; ++q) {
                            if (li[q] >= local_to_node[b].size() || local_to_node[b][li[q]] != dn[q])
                                fail("local index does not name the constraint's node");
                            if (owner[dn[q]] != b) fail("constraint node outside the CTA patch");
                            if (stamp[dn[q]] == epoch) fail("stage is not node-disjoint");
                            stamp[dn[q]] = epoch;
                            if (level > 0) outside[dn[q]] = 1;
                        }
                    }
                }
            }
        }
    }
    for (int k = 0; k < kKinds; ++k) {
        const GlobalTable& T = S.global[k];
        const int colours = T.colour_offsets.empty() ? 0 : static_cast<int>(T.colour_offsets.size()) - 1;
        for (int c = 0; c < colours; ++c) {
            ++epoch;
            for (uint32_t i = T.colour_offsets[c]; i < T.colour_offsets[c + 1]; ++i) {
                uint32_t dn[4];
                const int cnt = nodes_of(k, T.def_index[i], dn);
                ++seen[k][T.def_index[i]];
                const uint32_t slots[4] = {T.a[i], T.b[i], k ? T.c[i] : 0u, k ? T.d[i] : 0u};
                for (int q = 0; q < cnt; ++q) {
                    if (S.slot_of_node[dn[q]] != slots[q]) fail("global slot mismatch");
                    if (stamp[dn[q]] == epoch) fail("global colour is not node-disjoint");
                    stamp[dn[q]] = epoch;
                    outside[dn[q]] = 1;
                }
            }
        }
    }
    for (int k = 0; k < kKinds; ++k)
        for (size_t i = 0; i < seen[k].size(); ++i)
            if (seen[k][i] != 1) fail("constraint not scheduled exactly once");
    // seam stages: disjoint, and consistent with the sweep order
    const int seam_stages = S.seam_stage_offsets.empty() ? 0 : static_cast<int>(S.seam_stage_offsets.size()) - 1;
    for (int s = 0; s < seam_stages; ++s) {
        ++epoch;
        for (uint32_t i = S.seam_stage_offsets[s]; i < S.seam_stage_offsets[s + 1]; ++i)
            for (uint32_t slot : {S.seam_a[i], S.seam_b[i]}) {
                const uint32_t n = S.node_of_slot[slot];
                if (stamp[n] == epoch) fail("seam stage is not node-disjoint");
                stamp[n] = epoch;
                outside[n] = 1;
            }
    }
    // interface completeness
    std::vector<uint8_t> in_iface(N, 0);
    for (int b = 0; b < G; ++b)
        for (uint32_t i = S.iface_begin[b]; i < S.iface_begin[b + 1]; ++i)
            in_iface[S.node_of_slot[S.l1_begin[b] + S.iface_local[i]]] = 1;
    for (uint32_t n = 0; n < N; ++n)
        if (outside[n] && !in_iface[n]) fail("node touched outside level 1 is missing from the interface");
    // sweep orders are permutations in execution order
    for (int k = 0; k < kKinds; ++k) {
        const auto& order = k == 0 ? S.distance_order : S.dihedral_order;
        if (order.size() != seen[k].size()) fail("sweep order length");
    }
}

}  // namespace swb

namespace {
swb_status plan(const swb_structure_definition* definition, const swb_solver_options* options,
                swb_schedule_report* out, uint64_t* distance_order, uint64_t* dihedral_order,
                uint64_t* membrane_order);
}  // namespace

extern "C" swb_status swb_plan_schedule(const swb_structure_definition* definition,
                                        const swb_solver_options* options, swb_schedule_report* out,
                                        uint64_t* distance_order, uint64_t* dihedral_order) {
    return plan(definition, options, out, distance_order, dihedral_order, nullptr);
}

extern "C" swb_status swb_plan_membrane_order(const swb_structure_definition* definition,
                                              const swb_solver_options* options, uint64_t* membrane_order) {
    swb_schedule_report report;
    if (!membrane_order && definition && definition->membrane_count) return SWB_INVALID_ARGUMENT;
    return plan(definition, options, &report, nullptr, nullptr, membrane_order);
}

namespace {
swb_status plan(const swb_structure_definition* definition, const swb_solver_options* options,
                swb_schedule_report* out, uint64_t* distance_order, uint64_t* dihedral_order,
                uint64_t* membrane_order) {
    using namespace swb;
    return guarded([&] {
        if (!definition || !out) raise(SWB_INVALID_ARGUMENT, "null argument");
        OwnedDefinition def;
        def.assign(*definition);
        validate_definition(def.view);
        if (!(options && (options->flags & (SWB_OPT_GRID | SWB_OPT_GLOBAL_ONLY)))) {
            // Same choice as swb_structure_create, with the B200 opt-in
            // shared-memory budget (227 KB).
            const std::vector<uint32_t> susp = suspension_endpoint_nodes(def);
            const uint64_t N = def.nodes.size();
            int c = options && options->cluster_ctas > 0 ? options->cluster_ctas : 1;
            if (!(options && options->cluster_ctas > 0))
                while (c < kClusterMaxCtas && static_cast<uint64_t>(c) * 2048 < N) c *= 2;
            const int last = options && options->cluster_ctas > 0 ? c : kClusterMaxCtas;
            for (; c <= last; c *= 2) {
                ClusterSchedule C;
                if (!build_cluster_schedule(def, susp, c, C, options && (options->flags & SWB_OPT_SPLIT_STAGES)))
                    continue;
                const size_t bytes = cluster_shared_bytes(C);
                // opt-in shared memory less the kernels' static shared memory
                // (under 6 KB; the device build reads the exact figure)
                if (bytes > 227 * 1024 - 6144) continue;
                verify_cluster_schedule(def, susp, C);
                std::memset(out, 0, sizeof(*out));
                out->blocks = C.ctas;
                out->cluster_ctas = C.ctas;
                out->local_stages_per_iteration = total_stages(C);
                out->cluster_barriers_per_iteration = cluster_barriers_per_iteration(C);
                out->max_patch_nodes = static_cast<int32_t>(C.max_patch);
                out->shared_bytes = static_cast<int32_t>(bytes);
                out->level_constraints[0] = def.constraints.size() + def.dihedrals.size();
                if (distance_order) std::copy(C.distance_order.begin(), C.distance_order.end(), distance_order);
                if (dihedral_order) std::copy(C.dihedral_order.begin(), C.dihedral_order.end(), dihedral_order);
                if (membrane_order) std::copy(C.membrane_order.begin(), C.membrane_order.end(), membrane_order);
                return;
            }
            if (options && options->cluster_ctas > 0)
                raise(SWB_UNSUPPORTED, "the mesh does not fit the requested cluster");
        }
        ScheduleOptions so;
        so.blocks = options && options->blocks > 0 ? options->blocks : 148;
        so.blocks = static_cast<int>(std::min<uint64_t>(so.blocks, std::max<uint64_t>(1, def.nodes.size())));
        so.levels = options && options->partition_levels > 0 ? options->partition_levels : 3;
        so.global_only = options && (options->flags & SWB_OPT_GLOBAL_ONLY);
        const std::vector<uint32_t> susp = suspension_endpoint_nodes(def);
        const Schedule S = build_schedule(def, susp, so);
        verify_schedule(def, susp, S);
        std::memset(out, 0, sizeof(*out));
        out->blocks = S.blocks;
        out->partition_levels = S.levels;
        int phases = 0, stages = 0;
        for (int k = 0; k < kKinds; ++k) {
            bool outer = S.global[k].colour_offsets.size() > 1;
            for (int l = 0; l < S.levels; ++l) {
                stages += S.tables[l][k].stages;
                if (l > 0 && S.tables[l][k].stages > 0) { outer = true; ++phases; }
            }
            const int gc = S.global[k].colour_offsets.empty() ? 0 : static_cast<int>(S.global[k].colour_offsets.size()) - 1;
            out->global_colours_per_iteration += gc;
            phases += gc + (outer ? 1 : 0);
        }
        out->device_phases_per_iteration = phases;
        out->local_stages_per_iteration = stages;
        out->max_patch_nodes = S.max_patch_nodes;
        for (int l = 0; l < 4; ++l) out->level_constraints[l] = S.level_constraints[l];
        out->global_constraints = S.global_constraints;
        if (membrane_order && !def.membranes.empty())
            raise(SWB_UNSUPPORTED, "membrane elements need the cluster schedule");
        if (distance_order) std::copy(S.distance_order.begin(), S.distance_order.end(), distance_order);
        if (dihedral_order) std::copy(S.dihedral_order.begin(), S.dihedral_order.end(), dihedral_order);
    });
}
}  // namespace
