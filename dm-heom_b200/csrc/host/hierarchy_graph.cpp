// hierarchy_graph.cpp -- ADO hierarchy of the HEOM (host).
//
// Same node numbering as the reference (dm-heom/src/heom/hierarchy_graph.cpp:30-181):
// layer by layer from the top; within a layer the integer partitions of the
// layer depth in the order of integer_partition.cpp:41-106 (ascending
// lexicographic order of the non-increasing part sequences), each padded
// with zeros to the width, sorted ascending and expanded through its
// lexicographic permutations (std::next_permutation).  The tuple -> uid map
// is a lexicographic ranking of the tuples instead of a hash table.
#include <algorithm>
#include <numeric>

#include "heom_host.hpp"

namespace heomhost {

int64_t binomial(int64_t n, int64_t k)
{
    if (k < 0 || n < 0 || k > n) return 0;
    k = std::min(k, n - k);
    int64_t r = 1;
    for (int64_t i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

namespace {
void partitions_rec(int32_t remaining, int32_t max_part, int32_t s, std::vector<int32_t>& cur,
                    std::vector<int32_t>& out)
{
    if (remaining == 0) {
        if ((int32_t)cur.size() <= s) {
            for (int32_t p = 0; p < s; ++p) out.push_back(p < (int32_t)cur.size() ? cur[p] : 0);
        }
        return;
    }
    if ((int32_t)cur.size() >= s) return;
    for (int32_t p = 1; p <= std::min(remaining, max_part); ++p) {
        cur.push_back(p);
        partitions_rec(remaining - p, p, s, cur, out);
        cur.pop_back();
    }
}
} // namespace

std::vector<int32_t> integer_partitions(int32_t n, int32_t s)
{
    std::vector<int32_t> out, cur;
    if (n > 0 && s > 0) partitions_rec(n, n, s, cur, out);
    return out;
}

int64_t hierarchy_graph::lex_rank(const int32_t* t) const
{
    int64_t rank = 0;
    int64_t prefix = 0;
    for (int64_t k = 0; k < width_; ++k) {
        for (int32_t x = 0; x < t[k]; ++x) {
            const int64_t r = depth_ - prefix - x;
            if (r >= 0) rank += binom_[r + width_ - 1 - k][width_ - 1 - k];
        }
        prefix += t[k];
    }
    return rank;
}

hierarchy_graph::hierarchy_graph(int64_t width, int64_t depth) : width_(width), depth_(depth)
{
    if (width < 1 || depth < 1) throw config_error("hierarchy width and depth must be >= 1");
    nodes_ = binomial(width + depth, width);                         // :34
    first_non_plus_ = (int32_t)binomial(width + depth - 1, width);   // :40
    if (nodes_ > INT32_MAX) throw config_error("hierarchy too large for int32 uids");
    binom_.assign(width + depth + 2, std::vector<int64_t>(width + 2, 0));
    for (int64_t a = 0; a < width + depth + 2; ++a)
        for (int64_t b = 0; b < width + 2; ++b) binom_[a][b] = binomial(a, b);

    const size_t W = (size_t)width;
    tuples_.resize((size_t)nodes_ * W);
    nodes_per_depth_.assign(depth + 1, 0);
    std::vector<int32_t> uid_of_rank(nodes_, -1);
    int64_t uid = 0;
    std::vector<int32_t> t(W);
    for (int64_t d = 0; d <= depth; ++d) {
        std::vector<int32_t> parts = d == 0 ? std::vector<int32_t>(W, 0) : integer_partitions((int32_t)d, (int32_t)width);
        const size_t np = parts.size() / W;
        for (size_t p = 0; p < np; ++p) {
            std::copy(parts.begin() + p * W, parts.begin() + (p + 1) * W, t.begin());
            std::sort(t.begin(), t.end());
            do {
                std::copy(t.begin(), t.end(), tuples_.begin() + uid * W);
                uid_of_rank[lex_rank(t.data())] = (int32_t)uid;
                nodes_per_depth_[d]++;
                uid++;
            } while (std::next_permutation(t.begin(), t.end()));
        }
    }
    if (uid != nodes_) throw std::logic_error("hierarchy_graph: node count mismatch");

    // Neighbour ranks in O(1) each.  With prefix_k = t_0 + ... + t_{k-1} and
    // w_k = W-1-k, the rank is sum_k A_k(0) where
    //   A_k(d) = sum_{x < t_k} C(D - prefix_k - d - x + w_k, w_k)
    //          = C(D - prefix_k - d + w_k + 1, w_k + 1) - C(D - prefix_k - d - t_k + w_k + 1, w_k + 1)
    // (hockey stick).  Raising t_j shifts the prefixes after j by +1 (d = 1)
    // and adds one term at j; lowering it shifts them by -1 and drops one.
    plus_.assign((size_t)nodes_ * W, invalid_uid);
    minus_.assign((size_t)nodes_ * W, invalid_uid);
    auto C = [this](int64_t a, int64_t b) -> int64_t { return a < b || a < 0 ? 0 : binom_[a][b]; };
    std::vector<int64_t> prefix(W + 1), a0(W), pre0(W + 1), sufp(W + 1), sufm(W + 1);
    for (int64_t u = 0; u < nodes_; ++u) {
        const int32_t* tu = tuples_.data() + u * W;
        prefix[0] = 0;
        for (size_t k = 0; k < W; ++k) prefix[k + 1] = prefix[k] + tu[k];
        const int64_t sum = prefix[W];
        auto A = [&](size_t k, int64_t d) {
            const int64_t w = (int64_t)W - 1 - (int64_t)k, R = depth - prefix[k] - d;
            return C(R + w + 1, w + 1) - C(R - tu[k] + w + 1, w + 1);
        };
        pre0[0] = 0;
        for (size_t k = 0; k < W; ++k) {
            a0[k] = A(k, 0);
            pre0[k + 1] = pre0[k] + a0[k];
        }
        sufp[W] = sufm[W] = 0;
        for (size_t k = W; k-- > 0;) {
            sufp[k] = sufp[k + 1] + (sum < depth ? A(k, 1) : 0); // :151-156 (plus only below the last layer)
            sufm[k] = sufm[k + 1] + A(k, -1);
        }
        for (size_t j = 0; j < W; ++j) {
            const int64_t w = (int64_t)W - 1 - (int64_t)j, R = depth - prefix[j];
            if (sum < depth) // :151-156
                plus_[u * W + j] = uid_of_rank[pre0[j] + a0[j] + C(R - tu[j] + w, w) + sufp[j + 1]];
            if (tu[j] > 0) // :158-163
                minus_[u * W + j] = uid_of_rank[pre0[j] + a0[j] - C(R - tu[j] + 1 + w, w) + sufm[j + 1]];
        }
    }
}

std::vector<uint8_t> make_mask(const std::string& strategy, const hierarchy_graph& g, int32_t matsubaras,
                               int64_t first_layer)
{
    std::vector<uint8_t> mask((size_t)g.nodes(), 1); // MASK_TRUE
    if (strategy == "none") return mask;               // hierarchy_mask.cpp:37-45
    if (strategy != "single_excitation") throw config_error("unknown filtering strategy: " + strategy);
    // hierarchy_mask.cpp:48-110: keep an ADO when all its excitations sit on one bath
    const int64_t W = g.width();
    const int64_t baths = W / matsubaras;
    for (int64_t u = 0; u < g.nodes(); ++u) {
        const int32_t* t = g.tuples().data() + u * W;
        int64_t sum = 0;
        for (int64_t k = 0; k < W; ++k) sum += t[k];
        if (sum < first_layer) continue;
        bool found = false;
        for (int64_t b = 0; b < baths && !found; ++b) {
            int64_t bs = 0;
            for (int64_t k = b * matsubaras; k < (b + 1) * matsubaras; ++k) bs += t[k];
            found = bs == sum;
        }
        mask[u] = found ? 1 : 0;
    }
    return mask;
}

} // namespace heomhost
