// Host construction and checking of the cluster sweep schedule.
#include "cluster_schedule.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

namespace swb {

namespace {

uint32_t make_ref(const ClusterSchedule& s, uint32_t node) {
    const uint32_t slot = s.slot_of_node[node];
    const uint32_t cta = static_cast<uint32_t>(
        std::upper_bound(s.patch_begin.begin(), s.patch_begin.end(), slot) - s.patch_begin.begin() - 1);
    return (cta << 12) | (slot - s.patch_begin[cta]);
}

// Tries to colour with one colour fewer, repeatedly: the constraints of the
// last colour are spread over the others and the conflicts that causes are
// repaired by min-conflicts local search with a tabu list (each move puts a
// conflicting constraint into the colour with the fewest conflicts for it,
// not undoing a recent move unless that reaches a new best).  Stops at the
// first count it cannot reach within `budget` moves and keeps the last
// proper colouring.  Deterministic (fixed seed).  Returns the colour count.
int reduce_colours(const std::vector<std::array<uint32_t, 4>>& nodes, const std::vector<int>& counts,
                   uint32_t node_count, int colours, std::vector<int>& colour, long budget) {
    const size_t m = nodes.size();
    if (m == 0 || colours <= 1) return colours;
    // conflict graph (constraints sharing a node)
    std::vector<uint32_t> off(node_count + 1, 0);
    for (size_t i = 0; i < m; ++i)
        for (int q = 0; q < counts[i]; ++q) ++off[nodes[i][q] + 1];
    for (uint32_t v = 0; v < node_count; ++v) off[v + 1] += off[v];
    std::vector<uint32_t> inc(off.back());
    {
        std::vector<uint32_t> cur(off.begin(), off.end() - 1);
        for (size_t i = 0; i < m; ++i)
            for (int q = 0; q < counts[i]; ++q) inc[cur[nodes[i][q]]++] = static_cast<uint32_t>(i);
    }
    std::vector<uint32_t> nb_off(m + 1, 0), nb;
    {
        std::vector<uint32_t> tmp;
        for (size_t i = 0; i < m; ++i) {
            tmp.clear();
            for (int q = 0; q < counts[i]; ++q)
                for (uint32_t k = off[nodes[i][q]]; k < off[nodes[i][q] + 1]; ++k)
                    if (inc[k] != i) tmp.push_back(inc[k]);
            std::sort(tmp.begin(), tmp.end());
            tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
            nb.insert(nb.end(), tmp.begin(), tmp.end());
            nb_off[i + 1] = static_cast<uint32_t>(nb.size());
        }
    }
    uint64_t state = 0x9e3779b97f4a7c15ull;
    auto rnd = [&]() {
        state ^= state << 13;
        state ^= state >> 7;
        state ^= state << 17;
        return state;
    };
    // the constraints at one node form a clique: no colouring has fewer
    // colours than the largest incidence count
    uint32_t clique = 0;
    for (uint32_t v = 0; v < node_count; ++v) clique = std::max(clique, off[v + 1] - off[v]);
    for (int k = colours - 1; k >= static_cast<int>(std::max<uint32_t>(clique, 1)); --k) {
        std::vector<int> c2 = colour;
        for (size_t i = 0; i < m; ++i)
            if (c2[i] >= k) c2[i] = static_cast<int>(rnd() % k);
        std::vector<uint16_t> cnt(m * static_cast<size_t>(k), 0);
        for (size_t i = 0; i < m; ++i)
            for (uint32_t e = nb_off[i]; e < nb_off[i + 1]; ++e) ++cnt[i * k + c2[nb[e]]];
        long conflicts = 0;
        for (size_t i = 0; i < m; ++i) conflicts += cnt[i * k + c2[i]];
        conflicts /= 2;
        long best = conflicts;
        std::vector<long> tabu(m * static_cast<size_t>(k), 0);
        std::vector<uint32_t> open;
        std::vector<int64_t> pos(m, -1);
        auto update = [&](uint32_t i) {
            const bool bad = cnt[i * k + c2[i]] > 0;
            if (bad && pos[i] < 0) {
                pos[i] = static_cast<int64_t>(open.size());
                open.push_back(i);
            } else if (!bad && pos[i] >= 0) {
                const uint32_t last = open.back();
                open[pos[i]] = last;
                pos[last] = pos[i];
                open.pop_back();
                pos[i] = -1;
            }
        };
        for (size_t i = 0; i < m; ++i) update(static_cast<uint32_t>(i));
        for (long it = 0; it < budget && !open.empty(); ++it) {
            const uint32_t i = open[rnd() % open.size()];
            const int cur = c2[i];
            int bc = -1, bv = 1 << 30;
            for (int c = 0; c < k; ++c) {
                if (c == cur) continue;
                const int v = cnt[i * k + c];
                const bool aspiration = conflicts - cnt[i * k + cur] + v < best;
                if (tabu[i * k + c] > it && !aspiration) continue;
                if (v < bv || (v == bv && (rnd() & 1))) {
                    bv = v;
                    bc = c;
                }
            }
            if (bc < 0) continue;
            conflicts += bv - cnt[i * k + cur];
            tabu[i * k + cur] = it + 7 + static_cast<long>(rnd() % 10) + static_cast<long>(open.size() / 10);
            c2[i] = bc;
            for (uint32_t e = nb_off[i]; e < nb_off[i + 1]; ++e) {
                const uint32_t j = nb[e];
                --cnt[j * k + cur];
                ++cnt[j * k + bc];
                update(j);
            }
            update(i);
            best = std::min(best, conflicts);
        }
        if (!open.empty()) return k + 1;
        colour = c2;
        colours = k;
    }
    return colours;
}

// Evens out, CTA by CTA, how many records each colour gives the CTA, without
// adding colours: a constraint whose colour holds more than the CTA's mean
// moves to the colour with the fewest of the CTA's records that none of its
// conflicting constraints (shared nodes) has, as long as that colour holds
// at least two fewer.  Stages then carry similar record counts on every CTA,
// so the largest colours no longer need two rounds of the CTA's threads
// while the small ones leave them idle.
void balance_colours(const std::vector<std::array<uint32_t, 4>>& nodes, const std::vector<int>& counts,
                     const std::vector<int>& cta_of, int ctas, uint32_t node_count, int colours,
                     std::vector<int>& colour) {
    const size_t m = nodes.size();
    if (colours < 2 || colours > 64 || m == 0) return;
    std::vector<uint32_t> off(node_count + 1, 0);
    for (size_t i = 0; i < m; ++i)
        for (int q = 0; q < counts[i]; ++q) ++off[nodes[i][q] + 1];
    for (uint32_t v = 0; v < node_count; ++v) off[v + 1] += off[v];
    std::vector<uint32_t> inc(off.back());
    {
        std::vector<uint32_t> cur(off.begin(), off.end() - 1);
        for (size_t i = 0; i < m; ++i)
            for (int q = 0; q < counts[i]; ++q) inc[cur[nodes[i][q]]++] = static_cast<uint32_t>(i);
    }
    std::vector<int64_t> size(static_cast<size_t>(ctas) * colours, 0), total(ctas, 0);
    for (size_t i = 0; i < m; ++i) {
        ++size[static_cast<size_t>(cta_of[i]) * colours + colour[i]];
        ++total[cta_of[i]];
    }
    for (int pass = 0; pass < 8; ++pass) {
        bool moved = false;
        for (size_t i = 0; i < m; ++i) {
            const int c = colour[i];
            int64_t* sz = size.data() + static_cast<size_t>(cta_of[i]) * colours;
            const int64_t mean = (total[cta_of[i]] + colours - 1) / colours;
            if (sz[c] <= mean) continue;
            uint64_t used = 0;
            for (int q = 0; q < counts[i]; ++q)
                for (uint32_t k = off[nodes[i][q]]; k < off[nodes[i][q] + 1]; ++k)
                    if (inc[k] != i) used |= 1ull << colour[inc[k]];
            int best = -1;
            for (int t = 0; t < colours; ++t)
                if (!((used >> t) & 1ull) && sz[t] + 1 < sz[c] && (best < 0 || sz[t] < sz[best])) best = t;
            if (best < 0) continue;
            --sz[c];
            ++sz[best];
            colour[i] = best;
            moved = true;
        }
        if (!moved) break;
    }
}

}  // namespace

// Nodes of element i (definition index) of kind k: 2 (distance), 4
// (dihedral) or 3 (membrane: its triangle's corners); returns the count.
static int element_nodes(const OwnedDefinition& d, int k, size_t i, uint32_t* nodes) {
    if (k == 0) {
        nodes[0] = static_cast<uint32_t>(d.constraints[i].first_node);
        nodes[1] = static_cast<uint32_t>(d.constraints[i].second_node);
        return 2;
    }
    if (k == 1) {
        for (int q = 0; q < 4; ++q) nodes[q] = static_cast<uint32_t>(d.dihedrals[i].nodes[q]);
        return 4;
    }
    const swb_triangle_def& t = d.triangles[d.membranes[i].triangle];
    for (int q = 0; q < 3; ++q) nodes[q] = static_cast<uint32_t>(t.nodes[q]);
    return 3;
}

// Load-path order of the cables and ties (loadPathConstraintOrder,
// soft_body.cpp:528-629) in sweep order, then the level schedule of one
// cable pair (reverse pass, forward pass) over the distance records.
static void build_load_path(const OwnedDefinition& d, ClusterSchedule& S) {
    const size_t N = d.nodes.size();
    std::vector<uint8_t> structural(N, 0);
    std::vector<std::vector<uint32_t>> adj(N);
    for (size_t v = 0; v < N; ++v) structural[v] = d.nodes[v].fixed ? 1 : 0;
    for (const auto& t : d.triangles)
        for (int k = 0; k < 3; ++k) structural[t.nodes[k]] = 1;
    std::vector<uint64_t> seq;
    for (uint64_t i : S.distance_order) {  // the device sweep order
        const auto& c = d.constraints[i];
        if (c.kind == SWB_CONSTRAINT_DISTANCE || c.kind == SWB_CONSTRAINT_SEAM_STITCH) continue;
        seq.push_back(i);
    }
    for (const auto& c : d.constraints) {
        if (c.kind == SWB_CONSTRAINT_DISTANCE || c.kind == SWB_CONSTRAINT_SEAM_STITCH) {
            structural[c.first_node] = structural[c.second_node] = 1;
            continue;
        }
        adj[c.first_node].push_back(static_cast<uint32_t>(c.second_node));
        adj[c.second_node].push_back(static_cast<uint32_t>(c.first_node));
    }
    for (const auto& h : d.dihedrals)
        for (int k = 0; k < 4; ++k) structural[h.nodes[k]] = 1;
    S.pair_stages = 0;
    S.pair_offsets.assign(static_cast<size_t>(S.ctas), 0);
    S.pair_rec.clear();
    if (seq.empty()) return;
    // breadth-first depth from the structural skin; a component without a
    // structural node is rooted at its heaviest node (first of the smallest
    // inverse mass)
    const uint64_t unknown = ~uint64_t{0};
    std::vector<uint64_t> depth(N, unknown);
    std::vector<uint32_t> queue;
    for (size_t v = 0; v < N; ++v)
        if (structural[v] && !adj[v].empty()) {
            depth[v] = 0;
            queue.push_back(static_cast<uint32_t>(v));
        }
    size_t head = 0;
    for (;;) {
        while (head < queue.size()) {
            const uint32_t v = queue[head++];
            for (uint32_t u : adj[v])
                if (depth[u] == unknown) {
                    depth[u] = depth[v] + 1;
                    queue.push_back(u);
                }
        }
        size_t root = N;
        double smallest = std::numeric_limits<double>::infinity();
        for (size_t v = 0; v < N; ++v) {
            const double w = d.nodes[v].fixed ? 0.0 : 1.0 / d.nodes[v].mass;
            if (depth[v] == unknown && !adj[v].empty() && w < smallest) {
                root = v;
                smallest = w;
            }
        }
        if (root == N) break;
        depth[root] = 0;
        queue.push_back(static_cast<uint32_t>(root));
    }
    auto cdepth = [&](uint64_t i) {
        return std::max(depth[d.constraints[i].first_node], depth[d.constraints[i].second_node]);
    };
    std::stable_sort(seq.begin(), seq.end(), [&](uint64_t a, uint64_t b) { return cdepth(a) < cdepth(b); });
    // distance record and executing CTA of each definition index
    const ClusterKind& K = S.kinds[0];
    std::vector<uint32_t> rec_of(d.constraints.size(), ~0u);
    std::vector<int> cta_of_rec(K.def_index.size(), 0);
    for (int c = 0; c < S.ctas; ++c)
        for (uint32_t r = K.offsets[static_cast<size_t>(c) * (K.stages + 1)];
             r < K.offsets[static_cast<size_t>(c) * (K.stages + 1) + K.stages]; ++r) {
            rec_of[K.def_index[r]] = r;
            cta_of_rec[r] = c;
        }
    // levels of the reverse pass, then of the forward pass
    struct Item { int level, cta; uint32_t rec; };
    std::vector<Item> items;
    int levels = 0;
    for (int pass = 0; pass < 2; ++pass) {
        std::vector<int> last(N, -1);
        int top = -1;
        for (size_t k = 0; k < seq.size(); ++k) {
            const uint64_t i = pass == 0 ? seq[seq.size() - 1 - k] : seq[k];
            const auto& c = d.constraints[i];
            const int level = std::max(last[c.first_node], last[c.second_node]) + 1;
            last[c.first_node] = last[c.second_node] = level;
            top = std::max(top, level);
            items.push_back({levels + level, cta_of_rec[rec_of[i]], rec_of[i]});
        }
        levels += top + 1;
    }
    S.pair_stages = levels;
    std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) {
        if (a.cta != b.cta) return a.cta < b.cta;
        return a.level < b.level;
    });
    S.pair_offsets.assign(static_cast<size_t>(S.ctas) * (levels + 1), 0);
    size_t at = 0;
    for (int c = 0; c < S.ctas; ++c) {
        for (int l = 0; l <= levels; ++l) {
            while (at < items.size() && items[at].cta == c && items[at].level < l) ++at;
            S.pair_offsets[static_cast<size_t>(c) * (levels + 1) + l] = static_cast<uint32_t>(at);
        }
        while (at < items.size() && items[at].cta == c) ++at;
    }
    for (const Item& it : items) S.pair_rec.push_back(it.rec);
}

// True when a record of global stage g has a node flagged in `attached`.
static bool stage_touches(const OwnedDefinition& d, const ClusterSchedule& S, const std::vector<uint8_t>& attached,
                          int g) {
    int k, s;
    global_stage(S, g, k, s);
    const ClusterKind& K = S.kinds[k];
    for (int c = 0; c < S.ctas; ++c)
        for (uint32_t r = K.offsets[static_cast<size_t>(c) * (K.stages + 1) + s];
             r < K.offsets[static_cast<size_t>(c) * (K.stages + 1) + s + 1]; ++r) {
            uint32_t nodes[4];
            const int cnt = element_nodes(d, k, K.def_index[r], nodes);
            for (int q = 0; q < cnt; ++q)
                if (attached[nodes[q]]) return true;
        }
    return false;
}

bool build_cluster_schedule(const OwnedDefinition& d, const std::vector<uint32_t>& suspension_nodes, int ctas,
                            ClusterSchedule& S, bool split) {
    S = ClusterSchedule{};
    const uint32_t N = static_cast<uint32_t>(d.nodes.size());
    ctas = std::clamp(ctas, 1, kClusterMaxCtas);
    if (N == 0) ctas = 1;
    S.ctas = ctas;
    S.node_count = N;
    const std::vector<int> part = bisect_nodes(d, suspension_nodes, ctas, 0.03);
    S.patch_begin.assign(ctas + 1, 0);
    for (uint32_t n = 0; n < N; ++n) ++S.patch_begin[part[n] + 1];
    for (int c = 0; c < ctas; ++c) {
        S.max_patch = std::max(S.max_patch, S.patch_begin[c + 1]);
        S.patch_begin[c + 1] += S.patch_begin[c];
    }
    if (S.max_patch > kClusterPatchNodes) {
        S = ClusterSchedule{};
        return false;
    }
    S.node_of_slot.assign(N, 0);
    S.slot_of_node.assign(N, 0);
    {
        std::vector<uint32_t> cur(S.patch_begin.begin(), S.patch_begin.end() - 1);
        for (uint32_t n = 0; n < N; ++n) {
            const uint32_t s = cur[part[n]]++;
            S.node_of_slot[s] = n;
            S.slot_of_node[n] = s;
        }
    }
    if (!suspension_nodes.empty()) S.susp_cta = part[suspension_nodes[0]];

    for (int k = 0; k < 3; ++k) {
        ClusterKind& K = S.kinds[k];
        const size_t m = k == 0 ? d.constraints.size() : (k == 1 ? d.dihedrals.size() : d.membranes.size());
        std::vector<std::array<uint32_t, 4>> nodes(m);
        std::vector<int> counts(m, 0);
        for (size_t i = 0; i < m; ++i) {
            nodes[i] = {0, 0, 0, 0};
            counts[i] = element_nodes(d, k, i, nodes[i].data());
        }
        // executing CTA: owner of most of the constraint's nodes (ties: first)
        std::vector<int> cta_of(m, 0);
        std::vector<uint8_t> interior(m, 0);
        for (size_t i = 0; i < m; ++i) {
            int best = part[nodes[i][0]], best_count = 0;
            for (int q = 0; q < counts[i]; ++q) {
                int cnt = 0;
                for (int r = 0; r < counts[i]; ++r) cnt += part[nodes[i][r]] == part[nodes[i][q]];
                if (cnt > best_count) {
                    best_count = cnt;
                    best = part[nodes[i][q]];
                }
            }
            cta_of[i] = best;
            interior[i] = best_count == counts[i];
        }
        std::vector<int> colour(m, 0);  // becomes the stage
        if (!split || ctas == 1 || k == 2) {  // membranes: classic stages
            K.stages = dsatur_colour(nodes, counts, colour);
            K.stages = reduce_colours(nodes, counts, N, K.stages, colour, kColourSearchMoves);
            balance_colours(nodes, counts, cta_of, ctas, N, K.stages, colour);
            K.cluster_sync.assign(K.stages, 1);
            K.interior_stages = 0;
            K.boundary_stages = K.stages;
        } else {
            // Split stages.  A record whose nodes all lie in its CTA's patch
            // is interior; the others (boundary records) are coloured first
            // and alone, so they take only as many colours as the most
            // boundary records at one node need.  Interior records then
            // take the smallest colour free at all of their nodes,
            // boundary colours included, and open a colour of their own
            // only where none is.  The stages of interior-only colours run
            // first, each closed by a CTA barrier (a CTA touches its own
            // patch only), the last by a cluster barrier; every stage with
            // boundary records is closed by a cluster barrier.
            std::vector<size_t> ids;
            std::vector<std::array<uint32_t, 4>> sub;
            std::vector<int> subc;
            for (size_t i = 0; i < m; ++i)
                if (!interior[i]) {
                    ids.push_back(i);
                    sub.push_back(nodes[i]);
                    subc.push_back(counts[i]);
                }
            std::vector<int> col;
            int B = dsatur_colour(sub, subc, col);
            if (B > 1) B = reduce_colours(sub, subc, N, B, col, kColourSearchMoves);
            // colours in use at each node (bit c: colour c), boundary first
            std::vector<std::vector<uint64_t>> used(N);
            auto taken = [&](uint32_t n, int c) {
                const auto& u = used[n];
                return static_cast<size_t>(c >> 6) < u.size() && ((u[c >> 6] >> (c & 63)) & 1ull);
            };
            auto take = [&](uint32_t n, int c) {
                auto& u = used[n];
                if (u.size() <= static_cast<size_t>(c >> 6)) u.resize((c >> 6) + 1, 0ull);
                u[c >> 6] |= 1ull << (c & 63);
            };
            for (size_t j = 0; j < ids.size(); ++j) {
                colour[ids[j]] = col[j];
                for (int q = 0; q < subc[j]; ++q) take(sub[j][q], col[j]);
            }
            // interior records, most constrained first (largest node degree sum)
            std::vector<uint32_t> degree(N, 0);
            for (size_t i = 0; i < m; ++i)
                for (int q = 0; q < counts[i]; ++q) ++degree[nodes[i][q]];
            std::vector<size_t> inner;
            for (size_t i = 0; i < m; ++i)
                if (interior[i]) inner.push_back(i);
            auto weight = [&](size_t i) {
                uint32_t w = 0;
                for (int q = 0; q < counts[i]; ++q) w += degree[nodes[i][q]];
                return w;
            };
            std::stable_sort(inner.begin(), inner.end(), [&](size_t a, size_t b) { return weight(a) > weight(b); });
            int total = B;
            for (size_t i : inner) {
                int c = 0;
                for (;; ++c) {
                    bool free = true;
                    for (int q = 0; q < counts[i] && free; ++q) free = !taken(nodes[i][q], c);
                    if (free) break;
                }
                colour[i] = c;
                for (int q = 0; q < counts[i]; ++q) take(nodes[i][q], c);
                total = std::max(total, c + 1);
            }
            // stage order: interior-only colours, then the boundary colours
            std::vector<int> stage_of(total);
            const int inner_only = total - B;
            for (int c = 0; c < total; ++c) stage_of[c] = c >= B ? c - B : inner_only + c;
            for (size_t i = 0; i < m; ++i) colour[i] = stage_of[colour[i]];
            K.stages = total;
            K.interior_stages = inner_only;
            K.boundary_stages = B;
            K.cluster_sync.assign(K.stages, 1);
            for (int g = 0; g + 1 < inner_only; ++g) K.cluster_sync[g] = 0;
        }
        const int stages = K.stages;
        // records CTA-major, stage within, definition order within
        std::vector<uint32_t> idx(m);
        std::iota(idx.begin(), idx.end(), 0u);
        std::stable_sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) {
            if (cta_of[x] != cta_of[y]) return cta_of[x] < cta_of[y];
            return colour[x] < colour[y];
        });
        K.offsets.assign(static_cast<size_t>(ctas) * (stages + 1), 0);
        std::vector<uint32_t> count(static_cast<size_t>(ctas) * std::max(stages, 1), 0);
        for (size_t i = 0; i < m; ++i) ++count[static_cast<size_t>(cta_of[i]) * stages + colour[i]];
        uint32_t off = 0;
        for (int c = 0; c < ctas; ++c) {
            const uint32_t cta_start = off;
            for (int s = 0; s < stages; ++s) {
                K.offsets[static_cast<size_t>(c) * (stages + 1) + s] = off;
                off += count[static_cast<size_t>(c) * stages + s];
            }
            K.offsets[static_cast<size_t>(c) * (stages + 1) + stages] = off;
            K.max_cta_records = std::max(K.max_cta_records, off - cta_start);
        }
        for (uint32_t i : idx) {
            K.ab.push_back(make_ref(S, nodes[i][0]) | (make_ref(S, nodes[i][1]) << 16));
            if (k == 2) {
                K.cd.push_back(make_ref(S, nodes[i][2]));
                K.rest.push_back(0.0f);
                K.comp.push_back(0.0f);
            } else if (k == 1) {
                K.cd.push_back(make_ref(S, nodes[i][2]) | (make_ref(S, nodes[i][3]) << 16));
                K.rest.push_back(static_cast<float>(d.dihedrals[i].rest_angle));
                K.comp.push_back(static_cast<float>(d.dihedrals[i].compliance));
            } else {
                const auto& dc = d.constraints[i];
                const bool stitch = dc.kind == SWB_CONSTRAINT_SEAM_STITCH;
                K.rest.push_back(stitch ? 0.0f : static_cast<float>(dc.rest_length));
                float cp = stitch ? 0.0f : static_cast<float>(dc.compliance);
                if (dc.kind == SWB_CONSTRAINT_CABLE) cp = std::copysign(std::fabs(cp), -1.0f);
                K.comp.push_back(cp);
            }
            K.def_index.push_back(i);
        }
        // sweep order: stage-major, CTA, record order
        auto& order = k == 0 ? S.distance_order : (k == 1 ? S.dihedral_order : S.membrane_order);
        for (int s = 0; s < stages; ++s)
            for (int c = 0; c < ctas; ++c)
                for (uint32_t r = K.offsets[static_cast<size_t>(c) * (stages + 1) + s];
                     r < K.offsets[static_cast<size_t>(c) * (stages + 1) + s + 1]; ++r)
                    order.push_back(K.def_index[r]);
    }

    // line iteration window: the last two stages of the iteration, when
    // neither touches a suspension endpoint node (classic stages: both end in
    // a cluster barrier)
    if (S.susp_cta >= 0 && !(split && ctas > 1)) {
        std::vector<uint8_t> attached(N, 0);
        for (uint32_t n : suspension_nodes) attached[n] = 1;
        const int Sg = total_stages(S);
        if (Sg >= 2 && !stage_touches(d, S, attached, Sg - 2) && !stage_touches(d, S, attached, Sg - 1)) {
            S.line_stage = Sg - 2;
            for (int g = Sg - 2; g < Sg; ++g) {
                int k, s;
                global_stage(S, g, k, s);
                const ClusterKind& K = S.kinds[k];
                const size_t o = static_cast<size_t>(S.susp_cta) * (K.stages + 1) + s;
                S.line_owner_records = std::max(S.line_owner_records, K.offsets[o + 1] - K.offsets[o]);
            }
        }
    }

    build_load_path(d, S);

    // seam closing pass: level scheduling in sweep order, executing CTA =
    // owner of the first node
    {
        std::vector<int32_t> node_stage(N, -1);
        struct Rec { int stage, cta; uint64_t index; };
        std::vector<Rec> recs;
        for (uint64_t i : S.distance_order) {
            const auto& c = d.constraints[i];
            if (c.kind != SWB_CONSTRAINT_SEAM_STITCH) continue;
            const int s = std::max(node_stage[c.first_node], node_stage[c.second_node]) + 1;
            node_stage[c.first_node] = node_stage[c.second_node] = s;
            recs.push_back({s, part[c.first_node], i});
        }
        S.seam_stages = 0;
        for (const Rec& r : recs) S.seam_stages = std::max(S.seam_stages, r.stage + 1);
        std::stable_sort(recs.begin(), recs.end(), [](const Rec& x, const Rec& y) {
            if (x.cta != y.cta) return x.cta < y.cta;
            return x.stage < y.stage;
        });
        S.seam_offsets.assign(static_cast<size_t>(ctas) * (S.seam_stages + 1), 0);
        size_t at = 0;
        for (int c = 0; c < ctas; ++c) {
            for (int s = 0; s <= S.seam_stages; ++s) {
                while (at < recs.size() && recs[at].cta == c && recs[at].stage < s) ++at;
                S.seam_offsets[static_cast<size_t>(c) * (S.seam_stages + 1) + s] = static_cast<uint32_t>(at);
            }
            while (at < recs.size() && recs[at].cta == c) ++at;
        }
        for (const Rec& r : recs) {
            const auto& c = d.constraints[r.index];
            S.seam_ab.push_back(make_ref(S, static_cast<uint32_t>(c.first_node)) |
                                (make_ref(S, static_cast<uint32_t>(c.second_node)) << 16));
        }
    }
    return true;
}

void verify_cluster_schedule(const OwnedDefinition& d, const std::vector<uint32_t>& suspension_nodes,
                             const ClusterSchedule& S) {
    auto fail = [](const std::string& what) { raise(SWB_INVALID_ARGUMENT, "cluster schedule invariant: " + what); };
    const uint32_t N = static_cast<uint32_t>(d.nodes.size());
    const int C = S.ctas;
    if (C < 1 || C > kClusterMaxCtas) fail("cta count");
    if (S.patch_begin.size() != static_cast<size_t>(C) + 1 || S.patch_begin[C] != N) fail("patch ranges");
    for (uint32_t n = 0; n < N; ++n)
        if (S.node_of_slot[S.slot_of_node[n]] != n) fail("slot map");
    auto node_of_ref = [&](uint32_t ref) {
        const uint32_t cta = ref >> 12, local = ref & 0xfffu;
        if (static_cast<int>(cta) >= C || S.patch_begin[cta] + local >= S.patch_begin[cta + 1])
            fail("reference outside its patch");
        return S.node_of_slot[S.patch_begin[cta] + local];
    };
    for (uint32_t n : suspension_nodes) {
        const uint32_t slot = S.slot_of_node[n];
        if (slot < S.patch_begin[S.susp_cta] || slot >= S.patch_begin[S.susp_cta + 1])
            fail("suspension node outside the owner patch");
    }
    if (S.line_stage >= 0) {
        const int Sg = total_stages(S);
        if (S.susp_cta < 0 || S.line_stage != Sg - 2) fail("line iteration window position");
        std::vector<uint8_t> attached(N, 0);
        for (uint32_t n : suspension_nodes) attached[n] = 1;
        for (int g = Sg - 2; g < Sg; ++g) {
            int k, s;
            global_stage(S, g, k, s);
            if (stage_touches(d, S, attached, g)) fail("line iteration window touches a suspension node");
            if (!S.kinds[k].cluster_sync[s]) fail("line iteration window without cluster barriers");
            const size_t o = static_cast<size_t>(S.susp_cta) * (S.kinds[k].stages + 1) + s;
            if (S.kinds[k].offsets[o + 1] - S.kinds[k].offsets[o] > S.line_owner_records)
                fail("line iteration window record count");
        }
    }
    std::vector<int64_t> stamp(N, -1);
    int64_t epoch = 0;
    // runs of stages joined by CTA barriers: a node may be touched by one CTA only
    std::vector<int64_t> run_of(N, -1);
    std::vector<int> run_cta(N, -1);
    int64_t run = 0;
    for (int k = 0; k < 3; ++k) {
        const ClusterKind& K = S.kinds[k];
        const size_t m = k == 0 ? d.constraints.size() : (k == 1 ? d.dihedrals.size() : d.membranes.size());
        std::vector<uint8_t> seen(m, 0);
        if (K.cluster_sync.size() != static_cast<size_t>(K.stages)) fail("barrier kinds per stage");
        if (K.stages > 0 && !K.cluster_sync.back()) fail("a kind must end with a cluster barrier");
        for (int s = 0; s < K.stages; ++s) {
            ++epoch;
            for (int c = 0; c < C; ++c)
                for (uint32_t r = K.offsets[static_cast<size_t>(c) * (K.stages + 1) + s];
                     r < K.offsets[static_cast<size_t>(c) * (K.stages + 1) + s + 1]; ++r) {
                    const uint32_t i = K.def_index[r];
                    if (seen[i]++) fail("constraint scheduled twice");
                    const uint32_t refs[4] = {K.ab[r] & 0xffffu, K.ab[r] >> 16, k ? (K.cd[r] & 0xffffu) : 0u,
                                              k ? (K.cd[r] >> 16) : 0u};
                    uint32_t want[4];
                    const int cnt = element_nodes(d, k, i, want);
                    if (k == 2 && (K.cd[r] >> 16) != 0) fail("membrane record's fourth reference");
                    for (int q = 0; q < cnt; ++q) {
                        const uint32_t n = node_of_ref(refs[q]);
                        if (n != want[q]) fail("reference does not name the constraint's node");
                        if (stamp[n] == epoch) fail("stage is not node-disjoint");
                        stamp[n] = epoch;
                        if (run_of[n] == run && run_cta[n] != c)
                            fail("a node is touched by two CTAs between cluster barriers");
                        run_of[n] = run;
                        run_cta[n] = c;
                    }
                }
            if (K.cluster_sync[s]) ++run;
        }
        for (size_t i = 0; i < m; ++i)
            if (!seen[i]) fail("constraint not scheduled");
    }
    // cable pairs: node-disjoint levels, each record run by the CTA owning
    // it, every cable and tie once per pass
    {
        const ClusterKind& K = S.kinds[0];
        std::vector<int> owner_of(K.def_index.size(), -1);
        for (int c = 0; c < C; ++c)
            for (uint32_t r = K.offsets[static_cast<size_t>(c) * (K.stages + 1)];
                 r < K.offsets[static_cast<size_t>(c) * (K.stages + 1) + K.stages]; ++r)
                owner_of[r] = c;
        size_t load_path = 0;
        for (const auto& c : d.constraints)
            load_path += !(c.kind == SWB_CONSTRAINT_DISTANCE || c.kind == SWB_CONSTRAINT_SEAM_STITCH);
        if (S.pair_stages > 0 && S.pair_offsets.size() != static_cast<size_t>(C) * (S.pair_stages + 1))
            fail("pair offsets");
        if (S.pair_rec.size() != 2 * load_path) fail("every cable and tie once per pass of a pair");
        std::vector<uint8_t> visits(K.def_index.size(), 0);
        for (int l = 0; l < S.pair_stages; ++l) {
            ++epoch;
            for (int c = 0; c < C; ++c)
                for (uint32_t i = S.pair_offsets[static_cast<size_t>(c) * (S.pair_stages + 1) + l];
                     i < S.pair_offsets[static_cast<size_t>(c) * (S.pair_stages + 1) + l + 1]; ++i) {
                    const uint32_t r = S.pair_rec[i];
                    if (r >= K.def_index.size() || owner_of[r] != c) fail("pair record run by another CTA");
                    const auto& con = d.constraints[K.def_index[r]];
                    if (con.kind == SWB_CONSTRAINT_DISTANCE || con.kind == SWB_CONSTRAINT_SEAM_STITCH)
                        fail("pair record is not a cable or tie");
                    ++visits[r];
                    for (uint64_t n : {con.first_node, con.second_node}) {
                        if (stamp[n] == epoch) fail("pair level is not node-disjoint");
                        stamp[n] = epoch;
                    }
                }
        }
        for (size_t r = 0; r < visits.size(); ++r) {
            const auto& con = d.constraints[K.def_index[r]];
            const bool lp = !(con.kind == SWB_CONSTRAINT_DISTANCE || con.kind == SWB_CONSTRAINT_SEAM_STITCH);
            if (visits[r] != (lp ? 2 : 0)) fail("cable pair visits");
        }
    }
    for (int s = 0; s < S.seam_stages; ++s) {
        ++epoch;
        for (int c = 0; c < C; ++c)
            for (uint32_t r = S.seam_offsets[static_cast<size_t>(c) * (S.seam_stages + 1) + s];
                 r < S.seam_offsets[static_cast<size_t>(c) * (S.seam_stages + 1) + s + 1]; ++r)
                for (uint32_t ref : {S.seam_ab[r] & 0xffffu, S.seam_ab[r] >> 16}) {
                    const uint32_t n = node_of_ref(ref);
                    if (stamp[n] == epoch) fail("seam stage is not node-disjoint");
                    stamp[n] = epoch;
                }
    }
}

}  // namespace swb
