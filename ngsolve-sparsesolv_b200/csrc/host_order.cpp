// host_order.cpp -- see host_order.hpp.
#include "host_order.hpp"

#include <algorithm>
#include <numeric>

namespace ssv {

// The ABMC steps must match the reference exactly (the ordering decides the
// IC factor and hence the iteration count):
//   1. BFS aggregation: seeds are the lowest unassigned rows; the seed's
//      neighbours enter a FIFO (marked "queued"); rows are taken from the FIFO
//      until the block has block_size rows; rows still queued are released
//      (abmc_ordering.hpp:147-227).
//   2. Block graph: blocks adjacent through any nonzero (:235-273).
//   3. Greedy colouring of the block graph looking only at lower-numbered
//      neighbours, with at least max(target, max lower degree + 1) colours;
//      empty colours dropped (:288-353).
//   4. Rows numbered colour by colour, block by block (ascending block id),
//      rows of a block in ascending original index (:365-410).
void build_abmc(int n, const int* rp, const int* ci, int block_size, int target_colors,
                AbmcSchedule& out) {
    out = AbmcSchedule();
    if (n <= 0) return;
    if (block_size < 1) block_size = 1;
    if (target_colors < 2) target_colors = 2;
    const int max_blocks = (n + block_size - 1) / block_size;

    // 1. aggregation; block b owns members[first[b] .. first[b+1])
    std::vector<int> state(n, -1);  // -1 free, -2 queued, >= 0 block id
    std::vector<int> members;
    members.reserve(n);
    std::vector<int> first;
    first.reserve(max_blocks + 1);
    std::vector<int> fifo(n);
    int seed = 0;
    for (int b = 0; b < max_blocks; ++b) {
        while (seed < n && state[seed] >= 0) ++seed;
        if (seed >= n) break;
        const int id = static_cast<int>(first.size());
        first.push_back(static_cast<int>(members.size()));
        int size = 1;
        state[seed] = id;
        members.push_back(seed);
        int head = 0, tail = 0;
        auto enqueue_neighbours = [&](int row) {
            for (int k = rp[row]; k < rp[row + 1]; ++k) {
                const int j = ci[k];
                if (state[j] == -1) { state[j] = -2; fifo[tail++] = j; }
            }
        };
        enqueue_neighbours(seed);
        while (head < tail && size < block_size) {
            const int row = fifo[head++];
            if (state[row] >= 0) continue;
            state[row] = id;
            members.push_back(row);
            if (++size >= block_size) break;
            enqueue_neighbours(row);
        }
        for (; head < tail; ++head)
            if (state[fifo[head]] == -2) state[fifo[head]] = -1;
    }
    for (int i = 0; i < n; ++i) {
        if (state[i] < 0) {
            if (first.empty()) first.push_back(0);
            state[i] = static_cast<int>(first.size()) - 1;
            members.push_back(i);
        }
    }
    const int nb = static_cast<int>(first.size());
    first.push_back(static_cast<int>(members.size()));

    // 2. block adjacency
    std::vector<int> grp(nb + 1, 0), gci;
    gci.reserve(static_cast<size_t>(nb) * 12);
    std::vector<int> seen(nb, -1);
    for (int bi = 0; bi < nb; ++bi) {
        for (int m = first[bi]; m < first[bi + 1]; ++m) {
            const int row = members[m];
            for (int k = rp[row]; k < rp[row + 1]; ++k) {
                const int bj = state[ci[k]];
                if (bj != bi && seen[bj] != bi) { seen[bj] = bi; gci.push_back(bj); }
            }
        }
        grp[bi + 1] = static_cast<int>(gci.size());
    }

    // 3. greedy colouring
    int ncol = target_colors;
    for (int i = 0; i < nb; ++i) {
        int lower = 0;
        for (int k = grp[i]; k < grp[i + 1]; ++k) lower += (gci[k] < i);
        ncol = std::max(ncol, lower + 1);
    }
    std::vector<int> color(nb, -1), mark(ncol, -1);
    for (int i = 0; i < nb; ++i) {
        for (int k = grp[i]; k < grp[i + 1]; ++k) {
            const int j = gci[k];
            if (j < i) mark[color[j]] = i;
        }
        int c = 0;
        while (c < ncol && mark[c] == i) ++c;
        if (c == ncol) { ++ncol; mark.push_back(-1); }
        color[i] = c;
    }

    // 4. numbering; empty colours vanish
    std::vector<std::vector<int>> by_color(ncol);
    for (int b = 0; b < nb; ++b) by_color[color[b]].push_back(b);
    out.ordering.assign(n, 0);
    out.reverse.assign(n, 0);
    out.block_offsets.assign(nb + 1, 0);
    out.color_offsets.assign(1, 0);
    int next_row = 0, next_block = 0;
    for (int c = 0; c < ncol; ++c) {
        if (by_color[c].empty()) continue;
        for (int b : by_color[c]) {
            std::sort(members.begin() + first[b], members.begin() + first[b + 1]);
            out.block_offsets[next_block++] = next_row;
            for (int m = first[b]; m < first[b + 1]; ++m) {
                out.ordering[members[m]] = next_row;
                out.reverse[next_row] = members[m];
                ++next_row;
            }
        }
        out.color_offsets.push_back(next_block);
    }
    out.block_offsets[nb] = next_row;
    out.num_blocks = nb;
    out.num_colors = static_cast<int>(out.color_offsets.size()) - 1;
}

void rcm_order(int n, const int* rp, const int* ci, std::vector<int>& ordering, std::vector<int>& reverse) {
    ordering.assign(std::max(n, 0), 0);
    reverse.assign(std::max(n, 0), 0);
    if (n <= 0) return;
    std::vector<int> deg(n);
    for (int i = 0; i < n; ++i) deg[i] = rp[i + 1] - rp[i];
    int root = 0;
    for (int i = 1; i < n; ++i)
        if (deg[i] < deg[root]) root = i;
    // two sweeps toward a pseudo-peripheral row: the first row met at the
    // largest distance becomes the next root
    std::vector<int> dist(n);
    std::vector<int> fifo;
    fifo.reserve(n);
    for (int sweep = 0; sweep < 2; ++sweep) {
        std::fill(dist.begin(), dist.end(), -1);
        fifo.clear();
        fifo.push_back(root);
        dist[root] = 0;
        int far = root, far_d = 0;
        for (size_t h = 0; h < fifo.size(); ++h) {
            const int u = fifo[h];
            for (int k = rp[u]; k < rp[u + 1]; ++k) {
                const int v = ci[k];
                if (dist[v] >= 0) continue;
                dist[v] = dist[u] + 1;
                fifo.push_back(v);
                if (dist[v] > far_d) {
                    far_d = dist[v];
                    far = v;
                }
            }
        }
        root = far;
    }
    // Cuthill-McKee: breadth first, each row's unvisited neighbours by
    // ascending degree (std::sort with the same comparison, so rows of equal
    // degree land in the same order as the reference's)
    std::vector<char> seen(n, 0);
    std::vector<int> order;
    order.reserve(n);
    std::vector<int> nb;
    for (int s0 = 0; s0 < n; ++s0) {
        const int seed = s0 == 0 ? root : s0;
        if (seen[seed]) continue;
        seen[seed] = 1;
        const size_t head0 = order.size();
        order.push_back(seed);
        for (size_t h = head0; h < order.size(); ++h) {
            const int u = order[h];
            nb.clear();
            for (int k = rp[u]; k < rp[u + 1]; ++k) {
                const int v = ci[k];
                if (!seen[v]) {
                    seen[v] = 1;
                    nb.push_back(v);
                }
            }
            std::sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] < deg[b]; });
            for (int v : nb) order.push_back(v);
        }
    }
    for (int i = 0; i < n; ++i) {
        const int old = order[n - 1 - i];
        reverse[i] = old;
        ordering[old] = i;
    }
}

int build_levels(int n, const int* rp, const int* ci, bool upper, std::vector<int>& level_of) {
    level_of.assign(std::max(n, 0), 0);
    if (n <= 0) return 0;
    int maxl = 0;
    if (!upper) {
        for (int i = 0; i < n; ++i) {
            int dep = -1;
            for (int k = rp[i]; k < rp[i + 1]; ++k)
                if (ci[k] < i) dep = std::max(dep, level_of[ci[k]]);
            level_of[i] = dep + 1;
            maxl = std::max(maxl, level_of[i]);
        }
    } else {
        for (int i = n - 1; i >= 0; --i) {
            int dep = -1;
            for (int k = rp[i]; k < rp[i + 1]; ++k)
                if (ci[k] > i) dep = std::max(dep, level_of[ci[k]]);
            level_of[i] = dep + 1;
            maxl = std::max(maxl, level_of[i]);
        }
    }
    return maxl + 1;
}

void group_by_level(const std::vector<int>& level_of, int nlev, std::vector<int>& rows,
                    std::vector<int>& offsets) {
    const int n = static_cast<int>(level_of.size());
    offsets.assign(nlev + 1, 0);
    for (int i = 0; i < n; ++i) offsets[level_of[i] + 1]++;
    for (int l = 0; l < nlev; ++l) offsets[l + 1] += offsets[l];
    rows.assign(n, 0);
    std::vector<int> pos(offsets.begin(), offsets.end() - 1);
    for (int i = 0; i < n; ++i) rows[pos[level_of[i]]++] = i;
}

void permute_pattern(int n, const int* rp, const int* ci, const int* perm, std::vector<int>& prp,
                     std::vector<int>& pci, std::vector<int>& src) {
    prp.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) prp[perm[i] + 1] = rp[i + 1] - rp[i];
    for (int i = 0; i < n; ++i) prp[i + 1] += prp[i];
    const int nnz = prp[n];
    pci.assign(nnz, 0);
    src.assign(nnz, 0);
    std::vector<int> pos(prp.begin(), prp.end() - 1);
    for (int i = 0; i < n; ++i) {
        const int ni = perm[i];
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int p = pos[ni]++;
            pci[p] = perm[ci[k]];
            src[p] = k;
        }
    }
    // sort every row by column (insertion sort: rows are short)
    for (int i = 0; i < n; ++i) {
        for (int k = prp[i] + 1; k < prp[i + 1]; ++k) {
            const int c = pci[k], s = src[k];
            int m = k - 1;
            while (m >= prp[i] && pci[m] > c) { pci[m + 1] = pci[m]; src[m + 1] = src[m]; --m; }
            pci[m + 1] = c;
            src[m + 1] = s;
        }
    }
}

void lower_pattern(int n, const int* rp, const int* ci, std::vector<int>& lrp, std::vector<int>& lci,
                   std::vector<int>& lsrc) {
    lrp.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        int c = 0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) c += (ci[k] <= i);
        lrp[i + 1] = lrp[i] + c;
    }
    lci.resize(lrp[n]);
    lsrc.resize(lrp[n]);
    for (int i = 0; i < n; ++i) {
        int p = lrp[i];
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] <= i) { lci[p] = ci[k]; lsrc[p] = k; ++p; }
    }
}

void transpose_pattern(int n, const std::vector<int>& lrp, const std::vector<int>& lci,
                       std::vector<int>& urp, std::vector<int>& uci, std::vector<int>& usrc) {
    const int nnz = lrp[n];
    urp.assign(n + 1, 0);
    for (int k = 0; k < nnz; ++k) urp[lci[k] + 1]++;
    for (int i = 0; i < n; ++i) urp[i + 1] += urp[i];
    uci.assign(nnz, 0);
    usrc.assign(nnz, 0);
    std::vector<int> pos(urp.begin(), urp.end() - 1);
    for (int i = 0; i < n; ++i)
        for (int k = lrp[i]; k < lrp[i + 1]; ++k) {
            const int p = pos[lci[k]]++;
            uci[p] = i;
            usrc[p] = k;
        }
}

}  // namespace ssv
