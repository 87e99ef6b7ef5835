// Host-side row orders of square sparse matrices: reverse Cuthill-McKee
// (slq_rcm_order), row-group aggregation (slq_group_order), and the sampled
// statistics that decide whether to use them (slq_order_spread,
// slq_group_fill).  Validation and aggregation run on a small pool of host
// threads; every result is independent of the number of threads.
//
// Reverse Cuthill-McKee: breadth-first from the lowest-degree row of each
// component, the not-yet-visited neighbours of each visited row appended in
// increasing (degree, row), the visit order reversed.  The visited set is a
// bit table (32 KB for 2^18 rows), which keeps the edge loop in L1.
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
// as local as the base order made it.  Large orders run up to 8 such
// sweeps in parallel over segments of the base order (see aggregate).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <cstdint>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/slq.h"

namespace slq {
void set_error(const std::string& message);  // slq_engine.cu
}

namespace {

// Threads for the host orders: the machine's hardware threads, at most 16.
int host_threads()
{
    const unsigned h = std::thread::hardware_concurrency();
    return static_cast<int>(std::min(16u, std::max(1u, h)));
}

// A fixed set of threads that run one job at a time: run(f) calls f(t, n)
// on threads t = 0..n-1 (the caller is thread 0) and returns when all are
// done.  Idle workers spin briefly on the job counter before they block, so
// back-to-back jobs start within microseconds.
class Pool
{
  public:
    explicit Pool(int n) : n_(std::max(1, n))
    {
        for (int i = 1; i < n_; ++i) workers_.emplace_back([this, i] { loop(i); });
    }
    ~Pool()
    {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_.store(true);
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    Pool(const Pool&) = delete;
    Pool& operator=(const Pool&) = delete;

    int size() const { return n_; }

    void run(const std::function<void(int, int)>& f)
    {
        if (n_ == 1)
        {
            f(0, 1);
            return;
        }
        job_ = &f;
        pending_.store(n_ - 1, std::memory_order_relaxed);
        {
            std::lock_guard<std::mutex> g(m_);
            gen_.fetch_add(1, std::memory_order_release);
        }
        cv_.notify_all();
        f(0, n_);
        for (long spin = 0; pending_.load(std::memory_order_acquire) != 0; ++spin)
            if (spin > 4096) std::this_thread::yield();
        job_ = nullptr;
    }

  private:
    void loop(int i)
    {
        uint64_t seen = 0;
        for (;;)
        {
            long spin = 0;
            while (gen_.load(std::memory_order_acquire) == seen && !stop_.load() && spin < 200000)
                ++spin;
            if (gen_.load(std::memory_order_acquire) == seen && !stop_.load())
            {
                std::unique_lock<std::mutex> l(m_);
                cv_.wait(l, [&] { return stop_.load() || gen_.load() != seen; });
            }
            if (stop_.load()) return;
            seen = gen_.load(std::memory_order_acquire);
            (*job_)(i, n_);
            pending_.fetch_sub(1, std::memory_order_acq_rel);
        }
    }

    int n_;
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_;
    const std::function<void(int, int)>* job_ = nullptr;
    std::atomic<uint64_t> gen_{0};
    std::atomic<int> pending_{0};
    std::atomic<bool> stop_{false};
};

// The pool every entry point uses, created on first use and kept for the
// life of the process (its workers block when idle); one job at a time.
Pool& shared_pool()
{
    static Pool* pool = new Pool(host_threads());
    return *pool;
}

std::mutex& pool_mutex()
{
    static std::mutex m;
    return m;
}

// [begin, end) of part t of n of a range of `total` items
inline void part_range(int64_t total, int t, int n, int64_t& begin, int64_t& end)
{
    begin = total * t / n;
    end = total * (t + 1) / n;
}

// indptr starts non-negative and never decreases
bool valid_indptr(int64_t n, const int32_t* indptr, const char* who)
{
    if (indptr[0] < 0)
    {
        slq::set_error(std::string(who) + ": indptr[0] is negative");
        return false;
    }
    for (int64_t r = 0; r < n; ++r)
        if (indptr[r + 1] < indptr[r])
        {
            slq::set_error(std::string(who) + ": indptr is not monotone");
            return false;
        }
    return true;
}

// part t of nt of the check that every column index (of a pattern whose
// indptr passed valid_indptr) lies in [0, n): one unsigned comparison per
// index, or-ed without a branch so the loop vectorises (a negative index is
// a large unsigned one); true if this part holds a bad one
bool indices_out_of_range(int64_t n, const int32_t* indptr, const int32_t* indices, int t, int nt)
{
    const int64_t e0 = indptr[0], e1 = indptr[n];
    int64_t b, e;
    part_range(e1 - e0, t, nt, b, e);
    const uint32_t* ix = reinterpret_cast<const uint32_t*>(indices + e0);
    const uint32_t un = static_cast<uint32_t>(n);
    uint32_t any = 0;
    for (int64_t k = b; k < e; ++k) any |= static_cast<uint32_t>(ix[k] >= un);
    return any != 0;
}

void set_range_error(const char* who)
{
    slq::set_error(std::string(who) + ": column index out of range");
}

// indptr monotone from a non-negative start and every column index in
// [0, n): the checks that make the host loops below safe
bool valid_pattern(Pool& P, int64_t n, const int32_t* indptr, const int32_t* indices,
                   const char* who)
{
    if (!valid_indptr(n, indptr, who)) return false;
    std::atomic<bool> bad(false);
    P.run([&](int t, int nt) {
        if (indices_out_of_range(n, indptr, indices, t, nt))
            bad.store(true, std::memory_order_relaxed);
    });
    if (bad.load())
    {
        set_range_error(who);
        return false;
    }
    return true;
}

// row r's entries lie inside the index array (0 <= indptr[r] <= indptr[r+1]
// <= indptr[n]) and index [0, n): the checks a sampled row needs
bool valid_row(int64_t n, const int32_t* indptr, const int32_t* indices, int64_t r)
{
    if (indptr[r] < 0 || indptr[r + 1] < indptr[r] || indptr[r + 1] > indptr[n]) return false;
    for (int32_t e = indptr[r]; e < indptr[r + 1]; ++e)
        if (indices[e] < 0 || indices[e] >= n) return false;
    return true;
}

// inverse of a permutation, or false if perm is not one
bool inverse_perm(int64_t n, const int32_t* perm, std::vector<int32_t>& inv)
{
    inv.assign(static_cast<size_t>(n), -1);
    for (int64_t k = 0; k < n; ++k)
    {
        const int32_t r = perm[k];
        if (r < 0 || r >= n || inv[r] >= 0) return false;
        inv[r] = static_cast<int32_t>(k);
    }
    return true;
}

// The positions numpy's unique(linspace(0, last, count).astype(int64))
// gives: k * (last / (count - 1)) truncated, the last one exactly `last`.
std::vector<int64_t> sample_positions(int64_t last, int64_t count)
{
    std::vector<int64_t> out;
    if (count <= 0) return out;
    if (count == 1)
    {
        out.push_back(0);
        return out;
    }
    const double step = static_cast<double>(last) / static_cast<double>(count - 1);
    out.reserve(static_cast<size_t>(count));
    for (int64_t k = 0; k < count; ++k)
    {
        const int64_t v =
            (k == count - 1) ? last : static_cast<int64_t>(static_cast<double>(k) * step);
        if (out.empty() || v != out.back()) out.push_back(v);
    }
    return out;
}

// ---------------------------------------------------------------------------
// reverse Cuthill-McKee
// ---------------------------------------------------------------------------

// visited rows, one bit each
struct Bits {
    std::vector<uint64_t> w;
    explicit Bits(int64_t n) : w(static_cast<size_t>((n + 63) / 64), 0) {}
    bool get(int32_t r) const { return (w[static_cast<size_t>(r) >> 6] >> (r & 63)) & 1u; }
    void set(int32_t r) { w[static_cast<size_t>(r) >> 6] |= uint64_t(1) << (r & 63); }
};

// Cuthill-McKee visit order of every component into out[0 .. n)
void cm_order(int64_t n, const int32_t* indptr, const int32_t* indices, std::vector<int32_t>& out)
{
    std::vector<int32_t> degree(static_cast<size_t>(n));
    int32_t maxdeg = 0;
    for (int64_t r = 0; r < n; ++r)
    {
        degree[r] = indptr[r + 1] - indptr[r];
        maxdeg = std::max(maxdeg, degree[r]);
    }
    // rows by increasing degree, ties by row (a stable counting sort):
    // component start candidates
    std::vector<int32_t> by_degree(static_cast<size_t>(n));
    if (maxdeg <= 4 * n + 1024)
    {
        std::vector<int64_t> start(static_cast<size_t>(maxdeg) + 2, 0);
        for (int64_t r = 0; r < n; ++r) ++start[degree[r] + 1];
        for (size_t d = 1; d < start.size(); ++d) start[d] += start[d - 1];
        for (int64_t r = 0; r < n; ++r) by_degree[start[degree[r]]++] = static_cast<int32_t>(r);
    }
    else
    {
        for (int64_t r = 0; r < n; ++r) by_degree[r] = static_cast<int32_t>(r);
        std::stable_sort(by_degree.begin(), by_degree.end(),
                         [&](int32_t a, int32_t b) { return degree[a] < degree[b]; });
    }
    Bits visited(n);
    out.assign(static_cast<size_t>(n), 0);
    int64_t cnt = 0;
    std::vector<std::pair<int32_t, int32_t>> kids;
    for (int32_t seed : by_degree)
    {
        if (visited.get(seed)) continue;
        // each component starts at its lowest-degree row (as scipy's
        // reverse_cuthill_mckee does)
        int64_t head = cnt;
        out[cnt++] = seed;
        visited.set(seed);
        while (head < cnt)
        {
            const int32_t r = out[head++];
            kids.clear();
            for (int32_t e = indptr[r]; e < indptr[r + 1]; ++e)
            {
                const int32_t c = indices[e];
                if (!visited.get(c))
                {
                    visited.set(c);
                    kids.emplace_back(degree[c], c);
                }
            }
            std::sort(kids.begin(), kids.end());
            for (const auto& k : kids) out[cnt++] = k.second;
        }
    }
}

// ---------------------------------------------------------------------------
// row-group aggregation
// ---------------------------------------------------------------------------

// Candidate strength as one integer: |a_ij| rounded to float (the bits of a
// non-negative float order like its value) above, the complement of the row
// below, so that a larger key is a larger |a_ij|, then a smaller row.
inline uint64_t strength_key(float a, int32_t row)
{
    uint32_t bits;
    const float m = std::fabs(a);
    std::memcpy(&bits, &m, sizeof(bits));
    return (static_cast<uint64_t>(bits) << 32) | static_cast<uint32_t>(~static_cast<uint32_t>(row));
}

// Groups found by one sweep: their rows (G each, the last possibly fewer)
// and the base position of each group's seed.
struct Groups {
    std::vector<int32_t> rows;
    std::vector<int64_t> seed_pos;
};

// Rows a sweep may place: state[row] == me (the rows this sweep owns and has
// not placed yet; placing stores 0).  Other sweeps' rows are read, never
// written, so `state` is relaxed atomics.
struct SweepOwner {
    std::atomic<uint8_t>* state;
    uint8_t me;
    bool mine(int32_t r) const { return state[r].load(std::memory_order_relaxed) == me; }
    void take(int32_t r) const { state[r].store(0, std::memory_order_relaxed); }
};

// Asks for row r's column indices and values ahead of their use: a sweep
// visits rows in a data-dependent order, and a row whose cache lines arrive
// one miss at a time took most of the sweep's time.
template <typename VT>
inline void prefetch_row(const int32_t* indptr, const int32_t* indices, const VT* data, int32_t r)
{
    const int32_t e0 = indptr[r], e1 = indptr[r + 1];
    for (int32_t e = e0; e < e1; e += 16) __builtin_prefetch(indices + e);
    if (data)
        for (int32_t e = e0; e < e1; e += static_cast<int32_t>(64 / sizeof(VT)))
            __builtin_prefetch(data + e);
}

// One forward sweep over the seeds at base positions k0 .. seed_stop - 1
// (positions of `base`, NULL = identity) over the rows `own` lets it place.
// A group's seed takes its `want` strongest placeable neighbours (selected
// by strength_key), then theirs, and a group whose neighbourhood runs out is
// filled with the next placeable rows of base positions k0 .. stop - 1.
// A column index outside [0, n) is never placeable, so the sweep may run
// before, or beside, the check of the whole pattern's indices.
template <typename VT, typename Owner>
void aggregate_sweep(int64_t n, const int32_t* indptr, const int32_t* indices, const VT* data,
                     int G, const int32_t* base, int64_t k0, int64_t seed_stop, int64_t stop,
                     const Owner& own, Groups& out)
{
    const uint32_t un = static_cast<uint32_t>(n);
    const int step = 1;
    auto row_at = [&](int64_t k) { return base ? base[k] : static_cast<int32_t>(k); };
    auto mine = [&](int32_t r) { return own.mine(r); };
    auto take = [&](int32_t r) { own.take(r); };
    std::vector<int32_t> group, frontier, next;
    std::vector<uint64_t> keys;
    group.reserve(G);
    int64_t fill_cursor = k0;  // next sweep position for the fallback
    for (int64_t k = k0; k < seed_stop; k += step)
    {
        const int32_t seed = row_at(k);
        if (!mine(seed)) continue;
        group.clear();
        group.push_back(seed);
        take(seed);
        frontier.assign(1, seed);
        while (static_cast<int>(group.size()) < G && !frontier.empty())
        {
            next.clear();
            for (size_t i = 0; i < frontier.size(); ++i)
            {
                const int32_t f = frontier[i];
                const int want = G - static_cast<int>(group.size());
                if (want <= 0) break;
                if (i + 1 < frontier.size()) prefetch_row(indptr, indices, data, frontier[i + 1]);
                // every unplaced row of this sweep among f's neighbours, then
                // the `want` strongest of them
                const int32_t e0 = indptr[f], e1 = indptr[f + 1];
                keys.resize(static_cast<size_t>(e1 - e0));
                int m = 0;
                for (int32_t e = e0; e < e1; ++e)
                {
                    const int32_t c = indices[e];
                    const bool in = static_cast<uint32_t>(c) < un;
                    keys[m] = strength_key(data ? static_cast<float>(data[e]) : 1.0f, c);
                    m += (in && mine(in ? c : 0)) ? 1 : 0;
                }
                keys.resize(static_cast<size_t>(m));
                if (m > want)
                {
                    std::nth_element(keys.begin(), keys.begin() + want, keys.end(),
                                     std::greater<uint64_t>());
                    keys.resize(static_cast<size_t>(want));
                }
                std::sort(keys.begin(), keys.end(), std::greater<uint64_t>());
                for (uint64_t key : keys)
                {
                    const int32_t r = static_cast<int32_t>(~static_cast<uint32_t>(key));
                    if (!mine(r)) continue;  // a row that f lists twice joins once
                    take(r);
                    group.push_back(r);
                    next.push_back(r);
                }
            }
            frontier.swap(next);
        }
        while (static_cast<int>(group.size()) < G)
        {
            while (fill_cursor != stop && !mine(row_at(fill_cursor))) fill_cursor += step;
            if (fill_cursor == stop) break;
            const int32_t r = row_at(fill_cursor);
            take(r);
            group.push_back(r);
        }
        out.rows.insert(out.rows.end(), group.begin(), group.end());
        out.seed_pos.push_back(k);
    }
}

// Orders of at least 2 x 16384 rows are cut into K = min(8, n / 16384)
// segments of the base order; sweep s owns the rows whose base positions
// lie in segment s and runs forward through it (a row joins only the sweep
// that owns it), so the K sweeps are independent and run on the pool's
// threads in any assignment: the result does not depend on the number of
// threads.  Groups are listed by their seeds' base positions, the short
// groups at the segments' ends merged and put last.
//
// With `check`, the column indices of the whole pattern (whose indptr the
// caller has checked) are checked too: on the pool threads beyond the K
// sweeping ones, beside the sweeps, or before them when there are none.
// Returns false (the error set, `order` unspecified) for an index outside
// [0, n).
template <typename VT>
bool aggregate(Pool& P, int64_t n, const int32_t* indptr, const int32_t* indices, const VT* data,
               int G, const int32_t* base, const int32_t* base_pos, int32_t* order, bool check,
               const char* who)
{
    // state[r]: the sweep that owns unplaced row r (1 .. K), 0 once placed
    std::vector<std::atomic<uint8_t>> state(static_cast<size_t>(n));
    const int K = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(8, n / 16384)));
    const int64_t seg = (n + K - 1) / K;
    std::vector<Groups> sweep(static_cast<size_t>(K));
    P.run([&](int t, int nt) {
        int64_t b, e;
        part_range(n, t, nt, b, e);
        for (int64_t r = b; r < e; ++r)
        {
            const int64_t p = base_pos ? base_pos[r] : r;
            state[r].store(static_cast<uint8_t>(1 + p / seg), std::memory_order_relaxed);
        }
    });
    std::atomic<bool> bad(false);
    const bool beside = check && P.size() > K;
    if (check && !beside)
    {
        P.run([&](int t, int nt) {
            if (indices_out_of_range(n, indptr, indices, t, nt))
                bad.store(true, std::memory_order_relaxed);
        });
        if (bad.load())
        {
            set_range_error(who);
            return false;
        }
    }
    P.run([&](int t, int nt) {
        if (beside && t >= K)
        {
            if (indices_out_of_range(n, indptr, indices, t - K, nt - K))
                bad.store(true, std::memory_order_relaxed);
            return;
        }
        for (int s = t; s < K; s += beside ? K : nt)
        {
            const int64_t k0 = std::min<int64_t>(n, s * seg);
            const int64_t k1 = std::min<int64_t>(n, k0 + seg);
            aggregate_sweep<VT>(n, indptr, indices, data, G, base, k0, k1, k1,
                                SweepOwner{state.data(), static_cast<uint8_t>(s + 1)},
                                sweep[s]);
        }
    });
    if (bad.load())
    {
        set_range_error(who);
        return false;
    }
    struct Ref {
        int64_t seed_pos;
        int s;
        int64_t index;
    };
    std::vector<Ref> refs;
    std::vector<int32_t> tail;  // rows of the short groups
    for (int s = 0; s < static_cast<int>(sweep.size()); ++s)
    {
        const int64_t ng = static_cast<int64_t>(sweep[s].seed_pos.size());
        for (int64_t i = 0; i < ng; ++i)
        {
            const int64_t b = i * G;
            const int64_t e = std::min<int64_t>(b + G, static_cast<int64_t>(sweep[s].rows.size()));
            if (e - b < G)
                tail.insert(tail.end(), sweep[s].rows.begin() + b, sweep[s].rows.begin() + e);
            else
                refs.push_back(Ref{sweep[s].seed_pos[i], s, i});
        }
    }
    std::sort(refs.begin(), refs.end(),
              [](const Ref& a, const Ref& b) { return a.seed_pos < b.seed_pos; });
    int64_t out = 0;
    for (const Ref& rf : refs)
        for (int64_t i = rf.index * G; i < rf.index * G + G; ++i) order[out++] = sweep[rf.s].rows[i];
    for (int32_t r : tail) order[out++] = r;
    return true;
}

// Rows of the block being split: the thread's own bit per matrix row (set
// for the block's rows, cleared after) and, where the bit is set, the row's
// index in the block (loc) and its placed flag.
struct BlockOwner {
    const uint64_t* member;
    const int16_t* loc;
    uint8_t* placed;
    bool mine(int32_t r) const
    {
        return ((member[r >> 6] >> (r & 63)) & 1) && !placed[loc[r]];
    }
    void take(int32_t r) const { placed[loc[r]] = 1; }
};

// Blocks of B rows by aggregate(), then every whole block split into groups
// of G rows by the same sweep over its rows in base order, with the block's
// rows as the placeable ones.  Blocks run in parallel, each thread with its
// own membership bits and index table.
template <typename VT>
bool block_groups(Pool& P, int64_t n, const int32_t* indptr, const int32_t* indices,
                  const VT* data, int B, int G, const int32_t* base, const int32_t* base_pos,
                  int32_t* order, const char* who)
{
    if (!aggregate<VT>(P, n, indptr, indices, data, B, base, base_pos, order, true, who))
        return false;
    const int64_t nb = n / B;  // whole blocks; the rest stay last as they are
    P.run([&](int t, int nt) {
        int64_t b0, b1;
        part_range(nb, t, nt, b0, b1);
        if (b0 >= b1) return;
        std::vector<int32_t> rows(static_cast<size_t>(B));
        std::vector<uint64_t> member(static_cast<size_t>((n + 63) / 64), 0);
        std::unique_ptr<int16_t[]> loc(new int16_t[static_cast<size_t>(n)]);
        std::vector<uint8_t> placed(static_cast<size_t>(B));
        Groups g;
        for (int64_t b = b0; b < b1; ++b)
        {
            int32_t* blk = order + b * B;
            // the next block's rows load while this one is split
            if (b + 1 < b1)
                for (int i = 0; i < B; ++i) prefetch_row(indptr, indices, data, blk[B + i]);
            std::copy(blk, blk + B, rows.begin());
            if (base_pos)
                std::sort(rows.begin(), rows.end(),
                          [&](int32_t x, int32_t y) { return base_pos[x] < base_pos[y]; });
            else
                std::sort(rows.begin(), rows.end());
            for (int i = 0; i < B; ++i)
            {
                member[rows[i] >> 6] |= uint64_t(1) << (rows[i] & 63);
                loc[rows[i]] = static_cast<int16_t>(i);
            }
            std::fill(placed.begin(), placed.end(), 0);
            g.rows.clear();
            g.seed_pos.clear();
            aggregate_sweep<VT>(n, indptr, indices, data, G, rows.data(), 0, B, B,
                                BlockOwner{member.data(), loc.get(), placed.data()}, g);
            std::copy(g.rows.begin(), g.rows.end(), blk);
            for (int i = 0; i < B; ++i) member[rows[i] >> 6] = 0;
        }
    });
    return true;
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
    std::lock_guard<std::mutex> lock(pool_mutex());
    Pool& P = shared_pool();
    if (!valid_pattern(P, n, indptr, indices, "rcm_order")) return SLQ_ERR_BAD_CSR;
    std::vector<int32_t> out;
    cm_order(n, indptr, indices, out);
    // reverse Cuthill-McKee
    for (int64_t k = 0; k < n; ++k) order[k] = out[static_cast<size_t>(n - 1 - k)];
    return SLQ_OK;
}

extern "C" slq_status slq_group_order(int64_t n, const int32_t* indptr, const int32_t* indices,
                                      const void* data, int dtype, int group_rows,
                                      const int32_t* base_order, int32_t* order)
{
    if (n < 0 || !indptr || !indices || !order || group_rows < 1 || group_rows > 1024)
    {
        slq::set_error("group_order: bad arguments");
        return SLQ_ERR_BAD_ARG;
    }
    std::lock_guard<std::mutex> lock(pool_mutex());
    Pool& P = shared_pool();
    if (!valid_indptr(n, indptr, "group_order")) return SLQ_ERR_BAD_CSR;
    std::vector<int32_t> base_pos;
    if (base_order && !inverse_perm(n, base_order, base_pos))
    {
        slq::set_error("group_order: base_order is not a permutation");
        return SLQ_ERR_BAD_ARG;
    }
    const int32_t* bp = base_order ? base_pos.data() : nullptr;
    // the column indices are checked beside the sweeps
    const bool ok =
        dtype == SLQ_F64
            ? aggregate<double>(P, n, indptr, indices, static_cast<const double*>(data),
                                group_rows, base_order, bp, order, true, "group_order")
            : aggregate<float>(P, n, indptr, indices, static_cast<const float*>(data),
                               group_rows, base_order, bp, order, true, "group_order");
    return ok ? SLQ_OK : SLQ_ERR_BAD_CSR;
}

extern "C" slq_status slq_block_group_order(int64_t n, const int32_t* indptr,
                                            const int32_t* indices, const void* data, int dtype,
                                            int block_rows, int group_rows,
                                            const int32_t* base_order, int32_t* order)
{
    if (n < 0 || !indptr || !indices || !order || group_rows < 1 || group_rows > 1024 ||
        block_rows < group_rows || block_rows > 16384 || block_rows % group_rows != 0)  // int16 loc
    {
        slq::set_error("block_group_order: bad arguments");
        return SLQ_ERR_BAD_ARG;
    }
    std::lock_guard<std::mutex> lock(pool_mutex());
    Pool& P = shared_pool();
    if (!valid_indptr(n, indptr, "block_group_order")) return SLQ_ERR_BAD_CSR;
    std::vector<int32_t> base_pos;
    if (base_order && !inverse_perm(n, base_order, base_pos))
    {
        slq::set_error("block_group_order: base_order is not a permutation");
        return SLQ_ERR_BAD_ARG;
    }
    const int32_t* bp = base_order ? base_pos.data() : nullptr;
    // the column indices are checked beside the block sweeps
    const bool ok =
        dtype == SLQ_F64
            ? block_groups<double>(P, n, indptr, indices, static_cast<const double*>(data),
                                   block_rows, group_rows, base_order, bp, order,
                                   "block_group_order")
            : block_groups<float>(P, n, indptr, indices, static_cast<const float*>(data),
                                  block_rows, group_rows, base_order, bp, order,
                                  "block_group_order");
    return ok ? SLQ_OK : SLQ_ERR_BAD_CSR;
}

extern "C" slq_status slq_block_order(int64_t n, const int32_t* indptr, const int32_t* indices,
                                      const int32_t* group_order, int group_rows,
                                      int groups_per_block, int32_t* order)
{
    if (n < 0 || !indptr || !indices || !group_order || !order || group_rows < 1 ||
        group_rows > 1024 || groups_per_block < 1 || groups_per_block > 1024)
    {
        slq::set_error("block_order: bad arguments");
        return SLQ_ERR_BAD_ARG;
    }
    std::lock_guard<std::mutex> lock(pool_mutex());
    Pool& P = shared_pool();
    if (!valid_pattern(P, n, indptr, indices, "block_order")) return SLQ_ERR_BAD_CSR;
    std::vector<int32_t> pos;
    if (!inverse_perm(n, group_order, pos))
    {
        slq::set_error("block_order: group_order is not a permutation");
        return SLQ_ERR_BAD_ARG;
    }
    const int G = group_rows;
    const int64_t ng = n / G;  // whole groups; the remaining rows stay last
    // group of each row (-1: a row after the last whole group)
    std::vector<int32_t> gof(static_cast<size_t>(n), -1);
    for (int64_t k = 0; k < ng * G; ++k) gof[group_order[k]] = static_cast<int32_t>(k / G);
    // group graph: for each group, the groups its rows' neighbours fall in,
    // weighted by the number of such row pairs, and its own pair count
    std::vector<std::vector<std::pair<int32_t, int32_t>>> adj(static_cast<size_t>(ng));
    std::vector<int64_t> degree(static_cast<size_t>(ng), 0);
    P.run([&](int t, int nt) {
        int64_t b, e;
        part_range(ng, t, nt, b, e);
        std::vector<int32_t> cnt(b < e ? static_cast<size_t>(ng) : 0, 0);
        std::vector<int32_t> touched;
        for (int64_t g = b; g < e; ++g)
        {
            touched.clear();
            int64_t deg = 0;
            for (int r = 0; r < G; ++r)
            {
                const int32_t row = group_order[g * G + r];
                for (int32_t x = indptr[row]; x < indptr[row + 1]; ++x)
                {
                    const int32_t h = gof[indices[x]];
                    if (h < 0 || h == g) continue;
                    ++deg;
                    if (cnt[h]++ == 0) touched.push_back(h);
                }
            }
            degree[g] = deg;
            std::sort(touched.begin(), touched.end());
            adj[g].reserve(touched.size());
            for (int32_t h : touched)
            {
                adj[g].emplace_back(h, cnt[h]);
                cnt[h] = 0;
            }
        }
    });
    // greedy blocks on the graph: a seed group, then the unplaced neighbour
    // group with the most row pairs into the block per row pair of its own
    // (rows whose neighbours lie in the block share its columns); as good
    // as counting shared columns (same mean union on the benchmark matrix)
    // at a third of the cost
    std::vector<uint8_t> placed(static_cast<size_t>(ng), 0);
    std::vector<int64_t> grp_stamp(static_cast<size_t>(ng), -1);
    std::vector<int64_t> score(static_cast<size_t>(ng), 0);
    std::vector<int32_t> cand, block;
    int64_t out = 0, cursor = 0, bid = 0;
    auto join = [&](int64_t g) {
        placed[g] = 1;
        block.push_back(static_cast<int32_t>(g));
        for (const auto& hw : adj[g])
        {
            const int32_t h = hw.first;
            if (placed[h]) continue;
            if (grp_stamp[h] != bid)
            {
                grp_stamp[h] = bid;
                score[h] = 0;
                cand.push_back(h);
            }
            score[h] += hw.second;
        }
    };
    for (int64_t s = 0; s < ng; ++s, ++bid)
    {
        if (placed[s]) continue;
        block.clear();
        cand.clear();
        join(s);
        while (static_cast<int>(block.size()) < groups_per_block)
        {
            int64_t best = -1;
            for (int32_t h : cand)
            {
                if (placed[h]) continue;
                const int64_t lhs = score[h] * (best < 0 ? 1 : std::max<int64_t>(1, degree[best]));
                const int64_t rhs = (best < 0 ? -1 : score[best]) * std::max<int64_t>(1, degree[h]);
                if (best < 0 || lhs > rhs || (lhs == rhs && h < best)) best = h;
            }
            if (best < 0)
            {
                while (cursor < ng && placed[cursor]) ++cursor;
                if (cursor == ng) break;
                best = cursor;
            }
            join(best);
        }
        for (int32_t g : block)
            for (int r = 0; r < G; ++r) order[out++] = group_order[static_cast<int64_t>(g) * G + r];
    }
    for (int64_t k = ng * G; k < n; ++k) order[out++] = group_order[k];
    return SLQ_OK;
}

extern "C" slq_status slq_order_spread(int64_t n, const int32_t* indptr, const int32_t* indices,
                                       const int32_t* perm, int64_t sample_rows, double* spread)
{
    if (n < 0 || !indptr || !indices || !spread || sample_rows < 1)
    {
        slq::set_error("order_spread: bad arguments");
        return SLQ_ERR_BAD_ARG;
    }
    std::vector<int32_t> inv;
    if (perm && !inverse_perm(n, perm, inv))
    {
        slq::set_error("order_spread: perm is not a permutation");
        return SLQ_ERR_BAD_ARG;
    }
    *spread = 0.0;
    if (n == 0) return SLQ_OK;
    const std::vector<int64_t> rows = sample_positions(n - 1, std::min(n, sample_rows));
    // per-row sums in parallel (each sampled row checked first), added in
    // row order (thread-count independent)
    const int64_t m = static_cast<int64_t>(rows.size());
    std::vector<double> row_sum(static_cast<size_t>(m), 0.0);
    std::atomic<bool> bad(false);
    std::lock_guard<std::mutex> lock(pool_mutex());
    Pool& P = shared_pool();
    P.run([&](int t, int nt) {
        int64_t b, e;
        part_range(m, t, nt, b, e);
        for (int64_t i = b; i < e; ++i)
        {
            const int64_t r = rows[i];
            if (!valid_row(n, indptr, indices, r))
            {
                bad.store(true, std::memory_order_relaxed);
                return;
            }
            double sum = 0.0;
            for (int32_t x = indptr[r]; x < indptr[r + 1]; ++x)
            {
                const int64_t c = indices[x];
                const int64_t d = perm ? static_cast<int64_t>(inv[c]) - inv[r] : c - r;
                sum += static_cast<double>(d < 0 ? -d : d);
            }
            row_sum[i] = sum;
        }
    });
    if (bad.load())
    {
        slq::set_error("order_spread: bad CSR pattern");
        return SLQ_ERR_BAD_CSR;
    }
    double sum = 0.0;
    int64_t count = 0;
    for (int64_t i = 0; i < m; ++i)
    {
        sum += row_sum[i];
        count += indptr[rows[i] + 1] - indptr[rows[i]];
    }
    *spread = count ? sum / static_cast<double>(count) : 0.0;
    return SLQ_OK;
}

extern "C" slq_status slq_group_fill(int64_t n, const int32_t* indptr, const int32_t* indices,
                                     const int32_t* order, int group_rows, int64_t sample_groups,
                                     double* fill)
{
    if (n < 0 || !indptr || !indices || !fill || group_rows < 1 || sample_groups < 1)
    {
        slq::set_error("group_fill: bad arguments");
        return SLQ_ERR_BAD_ARG;
    }
    const int G = group_rows;
    const int64_t ngroups = n / G;
    *fill = 0.0;
    if (ngroups == 0) return SLQ_OK;
    const std::vector<int64_t> picks =
        sample_positions(ngroups - 1, std::min(sample_groups, ngroups));
    // per-group fills in parallel (each sampled row checked first), averaged
    // in group order
    const int64_t m = static_cast<int64_t>(picks.size());
    std::vector<double> ratio(static_cast<size_t>(m), -1.0);  // < 0: no entries
    std::atomic<bool> bad(false);
    std::lock_guard<std::mutex> lock(pool_mutex());
    Pool& P = shared_pool();
    P.run([&](int t, int nt) {
        int64_t b, e;
        part_range(m, t, nt, b, e);
        std::vector<int32_t> cols;
        std::vector<uint64_t> seen;  // bitmap over a group's column range
        for (int64_t i = b; i < e; ++i)
        {
            cols.clear();
            int32_t lo = INT32_MAX, hi = -1;
            for (int g = 0; g < G; ++g)
            {
                const int64_t k = picks[i] * G + g;
                const int32_t r = order ? order[k] : static_cast<int32_t>(k);
                if (r < 0 || r >= n || !valid_row(n, indptr, indices, r))
                {
                    bad.store(true, std::memory_order_relaxed);
                    return;
                }
                for (int32_t x = indptr[r]; x < indptr[r + 1]; ++x)
                {
                    lo = std::min(lo, indices[x]);
                    hi = std::max(hi, indices[x]);
                }
                cols.insert(cols.end(), indices + indptr[r], indices + indptr[r + 1]);
            }
            if (cols.empty()) continue;
            const int64_t nnz = static_cast<int64_t>(cols.size());
            // distinct columns: a bitmap over [lo, hi] when that is at most
            // 64 bits per entry, else sorting
            int64_t uni = 0;
            const int64_t words = (static_cast<int64_t>(hi) - lo) / 64 + 1;
            if (words <= nnz)
            {
                seen.assign(static_cast<size_t>(words), 0);
                for (const int32_t c : cols)
                    seen[static_cast<size_t>((c - lo) >> 6)] |= uint64_t(1) << ((c - lo) & 63);
                for (const uint64_t w : seen) uni += __builtin_popcountll(w);
            }
            else
            {
                std::sort(cols.begin(), cols.end());
                uni = std::unique(cols.begin(), cols.end()) - cols.begin();
            }
            ratio[i] = static_cast<double>(nnz) / (static_cast<double>(G) * static_cast<double>(uni));
        }
    });
    if (bad.load())
    {
        slq::set_error("group_fill: bad CSR pattern or order");
        return SLQ_ERR_BAD_CSR;
    }
    double sum = 0.0;
    int64_t ok = 0;
    for (int64_t i = 0; i < m; ++i)
        if (ratio[i] >= 0.0)
        {
            sum += ratio[i];
            ++ok;
        }
    *fill = ok ? sum / static_cast<double>(ok) : 0.0;
    return SLQ_OK;
}
