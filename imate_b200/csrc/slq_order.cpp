// Host-side row orders of square sparse matrices: reverse Cuthill-McKee
// (slq_rcm_order) and row-group aggregation (slq_group_order).
//
// Row-group aggregation:
// The row-group SpMM formats store, per group of G consecutive rows, the
// union of their columns with a dense value per (union column, row); their
// cost grows with the union, i.e. with how little the G rows' column sets
// overlap.  Consecutive rows of a bandwidth-reducing order (reverse
// Cuthill-McKee) form thin bands, so groups of them overlap poorly.  This
// order visits the rows in the base order and makes each not-yet-placed row
// the seed of a group: the seed, its strongest not-yet-placed neighbours
// (largest |a_ij| first -- for kernel matrices the nearest points), then
// their neighbours, and, if the neighbourhood is exhausted, the next
// not-yet-placed rows of the base order, so that every group except the
// last has exactly G rows and lines up with the device format's groups.
// Groups keep the base order's sequence, so the SpMM's gather window stays
// as local as the base order made it.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/slq.h"

namespace slq {
void set_error(const std::string& message);  // slq_engine.cu
}

namespace {

struct Cand {
    double w;
    int32_t row;
};

// a is stronger than b: larger |a_ij|, then the smaller row index
bool stronger(const Cand& a, const Cand& b)
{
    return a.w > b.w || (a.w == b.w && a.row < b.row);
}

template <typename VT>
void aggregate(int64_t n, const int32_t* indptr, const int32_t* indices, const VT* data, int G,
               const int32_t* base, int32_t* order)
{
    std::vector<uint8_t> placed(static_cast<size_t>(n), 0);
    std::vector<int32_t> group;
    std::vector<int32_t> frontier, next;
    std::vector<Cand> best;
    group.reserve(G);
    int64_t out = 0;
    int64_t fill_cursor = 0;  // next base position for the fallback
    for (int64_t k = 0; k < n; ++k)
    {
        const int32_t seed = base ? base[k] : static_cast<int32_t>(k);
        if (placed[seed]) continue;
        group.clear();
        group.push_back(seed);
        placed[seed] = 1;
        frontier.assign(1, seed);
        while (static_cast<int>(group.size()) < G && !frontier.empty())
        {
            next.clear();
            for (int32_t f : frontier)
            {
                const int want = G - static_cast<int>(group.size());
                if (want <= 0) break;
                // the `want` strongest unplaced neighbours of f: a heap whose
                // front is the weakest kept candidate
                best.clear();
                for (int32_t e = indptr[f]; e < indptr[f + 1]; ++e)
                {
                    const int32_t c = indices[e];
                    if (placed[c]) continue;
                    const double w = data ? std::fabs(static_cast<double>(data[e])) : 1.0;
                    const Cand cand{w, c};
                    if (static_cast<int>(best.size()) < want)
                    {
                        best.push_back(cand);
                        std::push_heap(best.begin(), best.end(), stronger);
                    }
                    else if (stronger(cand, best.front()))
                    {
                        std::pop_heap(best.begin(), best.end(), stronger);
                        best.back() = cand;
                        std::push_heap(best.begin(), best.end(), stronger);
                    }
                }
                std::sort(best.begin(), best.end(), stronger);
                for (const Cand& bc : best)
                {
                    placed[bc.row] = 1;
                    group.push_back(bc.row);
                    next.push_back(bc.row);
                }
            }
            frontier.swap(next);
        }
        while (static_cast<int>(group.size()) < G)
        {
            while (fill_cursor < n &&
                   placed[base ? base[fill_cursor] : static_cast<int32_t>(fill_cursor)])
                ++fill_cursor;
            if (fill_cursor >= n) break;
            const int32_t r = base ? base[fill_cursor] : static_cast<int32_t>(fill_cursor);
            placed[r] = 1;
            group.push_back(r);
        }
        for (int32_t r : group) order[out++] = r;
    }
}

// Breadth-first search from `start` over the unvisited rows of its
// component, the children of a row in increasing degree (Cuthill-McKee);
// appends the visit order to `out`.
void cm_bfs(int32_t start, const int32_t* indptr, const int32_t* indices, const int32_t* degree,
            std::vector<uint8_t>& visited, std::vector<int32_t>& out,
            std::vector<std::pair<int32_t, int32_t>>& kids)
{
    size_t head = out.size();
    out.push_back(start);
    visited[start] = 1;
    while (head < out.size())
    {
        const int32_t r = out[head++];
        kids.clear();
        for (int32_t e = indptr[r]; e < indptr[r + 1]; ++e)
        {
            const int32_t c = indices[e];
            if (!visited[c])
            {
                visited[c] = 1;
                kids.emplace_back(degree[c], c);
            }
        }
        std::sort(kids.begin(), kids.end());
        for (const auto& k : kids) out.push_back(k.second);
    }
}

}  // namespace

extern "C" slq_status slq_rcm_order(int64_t n, const int32_t* indptr, const int32_t* indices,
                                    int32_t* order)
{
    if (n < 0 || !indptr || !indices || !order)
    {
        slq::set_error("rcm_order: bad arguments");
        return SLQ_ERR_BAD_ARG;
    }
    for (int64_t r = 0; r < n; ++r)
        if (indptr[r + 1] < indptr[r])
        {
            slq::set_error("rcm_order: indptr is not monotone");
            return SLQ_ERR_BAD_CSR;
        }
    for (int64_t e = 0; e < indptr[n]; ++e)
        if (indices[e] < 0 || indices[e] >= n)
        {
            slq::set_error("rcm_order: column index out of range");
            return SLQ_ERR_BAD_CSR;
        }
    std::vector<int32_t> degree(static_cast<size_t>(n));
    for (int64_t r = 0; r < n; ++r) degree[r] = indptr[r + 1] - indptr[r];
    // rows by increasing degree: component start candidates
    std::vector<int32_t> by_degree(static_cast<size_t>(n));
    for (int64_t r = 0; r < n; ++r) by_degree[r] = static_cast<int32_t>(r);
    std::stable_sort(by_degree.begin(), by_degree.end(),
                     [&](int32_t a, int32_t b) { return degree[a] < degree[b]; });
    std::vector<uint8_t> visited(static_cast<size_t>(n), 0);
    std::vector<int32_t> out;
    std::vector<std::pair<int32_t, int32_t>> kids;
    out.reserve(static_cast<size_t>(n));
    for (int32_t seed : by_degree)
    {
        if (visited[seed]) continue;
        // each component starts at its lowest-degree row (as scipy's
        // reverse_cuthill_mckee does)
        const int32_t start = seed;
        cm_bfs(start, indptr, indices, degree.data(), visited, out, kids);
    }
    // reverse Cuthill-McKee
    for (int64_t k = 0; k < n; ++k) order[k] = out[static_cast<size_t>(n - 1 - k)];
    return SLQ_OK;
}

extern "C" slq_status slq_group_order(int64_t n, const int32_t* indptr, const int32_t* indices,
                                      const void* data, int dtype, int group_rows,
                                      const int32_t* base_order, int32_t* order)
{
    if (n < 0 || !indptr || !indices || !order || group_rows < 1 || group_rows > 32)
    {
        slq::set_error("group_order: bad arguments");
        return SLQ_ERR_BAD_ARG;
    }
    for (int64_t r = 0; r < n; ++r)
        if (indptr[r + 1] < indptr[r])
        {
            slq::set_error("group_order: indptr is not monotone");
            return SLQ_ERR_BAD_CSR;
        }
    for (int64_t e = 0; e < indptr[n]; ++e)
        if (indices[e] < 0 || indices[e] >= n)
        {
            slq::set_error("group_order: column index out of range");
            return SLQ_ERR_BAD_CSR;
        }
    if (base_order)
    {
        std::vector<uint8_t> seen(static_cast<size_t>(n), 0);
        for (int64_t k = 0; k < n; ++k)
        {
            const int32_t r = base_order[k];
            if (r < 0 || r >= n || seen[r])
            {
                slq::set_error("group_order: base_order is not a permutation");
                return SLQ_ERR_BAD_ARG;
            }
            seen[r] = 1;
        }
    }
    if (dtype == SLQ_F64)
        aggregate<double>(n, indptr, indices, static_cast<const double*>(data), group_rows,
                          base_order, order);
    else
        aggregate<float>(n, indptr, indices, static_cast<const float*>(data), group_rows,
                         base_order, order);
    return SLQ_OK;
}
