// Host setup for the device path: level sets and sweep schedules, and the
// node orderings of ordering.hpp.  Runs once per pattern (symbolic setup).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <numeric>
#include <queue>
#include <utility>
#include <vector>

#include "owtk_internal.h"

namespace owtk {

// Level of a row = 0 without a local dependency on the solved side, else
// 1 + the largest level among its dependencies.  Lower: columns < row
// (forward sweep); upper: row < column < owned (backward sweep).
void levels_of(std::size_t owned, const std::int32_t* rowptr, const std::int32_t* cols,
               std::vector<std::int32_t>& lower, std::vector<std::int32_t>& upper)
{
    lower.assign(owned, 0);
    upper.assign(owned, 0);
    const auto n = static_cast<std::int32_t>(owned);
    for (std::int32_t r = 0; r < n; ++r) {
        std::int32_t lv = 0;
        for (std::int32_t e = rowptr[r]; e < rowptr[r + 1]; ++e) {
            const std::int32_t c = cols[e];
            if (c < r) lv = std::max(lv, lower[c] + 1);
        }
        lower[r] = lv;
    }
    for (std::int32_t r = n - 1; r >= 0; --r) {
        std::int32_t lv = 0;
        for (std::int32_t e = rowptr[r]; e < rowptr[r + 1]; ++e) {
            const std::int32_t c = cols[e];
            if (c > r && c < n) lv = std::max(lv, upper[c] + 1);
        }
        upper[r] = lv;
    }
}

// Rows bucketed by level (ascending rows inside a level), cut into tasks of
// at most rows_per_task rows that never cross a level boundary.
void build_sweep(Context& ctx, Sweep& s, std::size_t owned, std::size_t bs,
                 const std::vector<std::int32_t>& level, bool /*descending_rows*/)
{
    s.h_level = level;
    s.rows_per_task = bs <= 32 ? static_cast<int>(32 / bs) : 1;
    std::int32_t depth = 0;
    for (const auto l : level) depth = std::max(depth, l + 1);
    s.depth = owned == 0 ? 0 : depth;
    std::vector<std::int32_t> count(static_cast<std::size_t>(depth) + 1, 0);
    for (const auto l : level) ++count[static_cast<std::size_t>(l) + 1];
    std::partial_sum(count.begin(), count.end(), count.begin());
    std::vector<std::int32_t> order(owned);
    {
        std::vector<std::int32_t> next(count.begin(), count.end() - 1);
        for (std::size_t r = 0; r < owned; ++r)
            order[static_cast<std::size_t>(next[static_cast<std::size_t>(level[r])]++)] =
                static_cast<std::int32_t>(r);
    }
    std::vector<std::int32_t> tasks{0};
    for (std::int32_t l = 0; l < depth; ++l) {
        for (std::int32_t p = count[static_cast<std::size_t>(l)]; p < count[static_cast<std::size_t>(l) + 1];
             p += s.rows_per_task) {
            tasks.push_back(std::min(p + s.rows_per_task, count[static_cast<std::size_t>(l) + 1]));
        }
    }
    s.tasks = static_cast<int>(tasks.size()) - 1;
    s.order = upload(ctx.stream, order);
    s.task_start = upload(ctx.stream, tasks);
    s.h_order = std::move(order);
}

// The factor entries an ILU sweep reads (lower entries for the forward sweep,
// upper for the backward, in the row's entry order), row after row in task
// order.  The rows of one level are scattered over the factor, and within a
// row the lower and upper entries sit side by side, so reading them in place
// fetches whole sectors for part of a row; packed, a task's entries are one
// contiguous run.  The values are gathered by every numeric factorisation.
void pack_sweep(Context& ctx, Sweep& s, std::size_t bs, std::size_t element_size,
                const std::vector<std::int32_t>& rowptr, const std::vector<std::int32_t>& cols,
                const std::vector<std::int32_t>& diagpos, bool backward)
{
    const std::size_t n = s.h_order.size();
    std::vector<std::int32_t> seg(n + 1, 0), pcols;
    std::vector<std::int64_t> psrc;
    pcols.reserve(cols.size() / 2 + 1);
    psrc.reserve(cols.size() / 2 + 1);
    for (std::size_t q = 0; q < n; ++q) {
        const std::size_t row = static_cast<std::size_t>(s.h_order[q]);
        const std::int32_t b = backward ? diagpos[row] + 1 : rowptr[row];
        const std::int32_t e = backward ? rowptr[row + 1] : diagpos[row];
        for (std::int32_t k = b; k < e; ++k) {
            pcols.push_back(cols[static_cast<std::size_t>(k)]);
            psrc.push_back(k);
        }
        seg[q + 1] = static_cast<std::int32_t>(pcols.size());
    }
    s.pentries = pcols.size();
    if (pcols.empty()) {
        pcols.push_back(0);
        psrc.push_back(0);
    }
    s.seg = upload(ctx.stream, seg);
    s.pcols = upload(ctx.stream, pcols);
    s.psrc = upload(ctx.stream, psrc);
    s.pvals.allocate(s.pentries * bs * element_size + 16);
    s.packed = true;
}

// ordering.hpp:138-180: BFS from the lowest-degree unvisited node, unvisited
// neighbours enqueued by ascending degree (std::sort with the same comparator,
// so ties resolve exactly as the reference's), and the order reversed.
void rcm_order(std::size_t owned, const std::int32_t* rowptr, const std::int32_t* cols,
               std::uint64_t* out)
{
    const std::size_t n = owned;
    std::vector<std::size_t> gptr(n + 1, 0);
    std::vector<std::size_t> adj;
    adj.reserve(static_cast<std::size_t>(rowptr[n]));
    for (std::size_t r = 0; r < n; ++r) {
        const std::size_t start = adj.size();
        for (std::int32_t e = rowptr[r]; e < rowptr[r + 1]; ++e) {
            const auto c = static_cast<std::size_t>(cols[e]);
            if (c < n && c != r) adj.push_back(c);
        }
        std::sort(adj.begin() + static_cast<std::ptrdiff_t>(start), adj.end());
        adj.erase(std::unique(adj.begin() + static_cast<std::ptrdiff_t>(start), adj.end()), adj.end());
        gptr[r + 1] = adj.size();
    }
    auto degree = [&](std::size_t v) { return gptr[v + 1] - gptr[v]; };
    std::vector<char> visited(n, 0);
    std::vector<std::size_t> order;
    order.reserve(n);
    std::vector<std::size_t> queue(n);
    std::vector<std::size_t> neighbors;
    while (order.size() < n) {
        std::size_t seed = n;
        for (std::size_t v = 0; v < n; ++v)
            if (!visited[v] && (seed == n || degree(v) < degree(seed))) seed = v;
        std::size_t head = 0, tail = 0;
        queue[tail++] = seed;
        visited[seed] = 1;
        while (head < tail) {
            const std::size_t v = queue[head++];
            order.push_back(v);
            neighbors.clear();
            for (std::size_t e = gptr[v]; e < gptr[v + 1]; ++e)
                if (!visited[adj[e]]) neighbors.push_back(adj[e]);
            std::sort(neighbors.begin(), neighbors.end(),
                      [&](std::size_t a, std::size_t b) { return degree(a) < degree(b); });
            for (const std::size_t u : neighbors) {
                if (!visited[u]) {
                    visited[u] = 1;
                    queue[tail++] = u;
                }
            }
        }
    }
    for (std::size_t i = 0; i < n; ++i) out[i] = order[n - 1 - i];
}

// ordering.hpp:51-77 and :231-261: Hilbert index of bounding-box-normalised
// coordinates on a 2^16 grid; sorted by (index, node).
void hilbert_order(std::size_t n, const double* xy, std::uint64_t* out)
{
    if (n == 0) return;
    double x0 = xy[0], x1 = xy[0], y0 = xy[1], y1 = xy[1];
    for (std::size_t i = 0; i < n; ++i) {
        x0 = std::min(x0, xy[2 * i]); x1 = std::max(x1, xy[2 * i]);
        y0 = std::min(y0, xy[2 * i + 1]); y1 = std::max(y1, xy[2 * i + 1]);
    }
    constexpr std::uint32_t extent = 1u << 16;
    const double eps = std::numeric_limits<double>::epsilon();
    std::vector<std::pair<std::uint64_t, std::size_t>> keyed(n);
    for (std::size_t i = 0; i < n; ++i) {
        const double nx = std::clamp((xy[2 * i] - x0) / std::max(x1 - x0, eps), 0.0, 1.0);
        const double ny = std::clamp((xy[2 * i + 1] - y0) / std::max(y1 - y0, eps), 0.0, 1.0);
        auto x = static_cast<std::uint32_t>(nx * (extent - 1));
        auto y = static_cast<std::uint32_t>(ny * (extent - 1));
        std::uint64_t index = 0;
        for (std::uint32_t s = extent / 2; s > 0; s /= 2) {
            const std::uint32_t rx = (x & s) != 0, ry = (y & s) != 0;
            index += static_cast<std::uint64_t>(s) * s * ((3u * rx) ^ ry);
            if (ry == 0) {
                if (rx == 1) { x = s - 1 - x; y = s - 1 - y; }
                std::swap(x, y);
            }
        }
        keyed[i] = {index, i};
    }
    std::sort(keyed.begin(), keyed.end());
    for (std::size_t i = 0; i < n; ++i) out[i] = keyed[i].second;
}

}  // namespace owtk
