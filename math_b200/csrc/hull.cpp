// Exact convex hull in 3..6 dimensions (nt_convex_hull, include/ntrace.h): the meshes of the measured
// scenes are boundaries of hulls of points on spheres.  As the reference's hull
// (src/geometry/core/convex_hull.cpp) the points are shuffled with std::mt19937_64(point count)
// (:667-670), scaled to integers in [0, 2^30 - 1] keeping proportions and rounded (:672-707),
// duplicates dropped, and the hull is built incrementally in that random order with exact integer
// predicates, so that no rounding decides a facet.  The algorithm here is the beneath-beyond
// insertion with outside sets: every point not yet inserted is assigned to one facet it sees; the
// next point's visible facets are found by a search from its facet over facet adjacency, replaced by
// the cone of new facets over the horizon ridges, and the orphaned points are reassigned among the
// new facets only (a point that saw a deleted facet and lies outside the new hull sees one of the new
// facets).  Hyperplanes are kept as exact integer normals (cofactors of the edge vectors) and offsets;
// 128-bit integers suffice up to 4 dimensions, 256-bit fixed-width integers are used above.
#include "ntrace.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <memory>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace ntrace
{
int report_error(int code, const std::string& message);
}

struct nt_hull
{
        int n = 0;
        std::vector<int32_t> facets;
};

namespace
{
// ---- 256-bit two's-complement integers (enough for 6-dimensional determinants of 30-bit values)

struct I256
{
        uint64_t w[4];
};

inline I256 i256(long long v)
{
        const uint64_t ext = v < 0 ? ~0ull : 0ull;
        return I256{{(uint64_t)v, ext, ext, ext}};
}

inline I256 operator+(const I256& a, const I256& b)
{
        I256 r;
        unsigned __int128 carry = 0;
        for (int i = 0; i < 4; ++i)
        {
                const unsigned __int128 s = (unsigned __int128)a.w[i] + b.w[i] + carry;
                r.w[i] = (uint64_t)s;
                carry = s >> 64;
        }
        return r;
}

inline I256 operator-(const I256& a)
{
        I256 r;
        unsigned __int128 carry = 1;
        for (int i = 0; i < 4; ++i)
        {
                const unsigned __int128 s = (unsigned __int128)(~a.w[i]) + carry;
                r.w[i] = (uint64_t)s;
                carry = s >> 64;
        }
        return r;
}

inline I256 operator-(const I256& a, const I256& b)
{
        return a + (-b);
}

inline bool negative(const I256& a)
{
        return (a.w[3] >> 63) != 0;
}

// low 256 bits of the product (exact while the true product fits, which the callers guarantee)
inline I256 operator*(const I256& x, const I256& y)
{
        const bool neg = negative(x) != negative(y);
        const I256 a = negative(x) ? -x : x;
        const I256 b = negative(y) ? -y : y;
        uint64_t r[4] = {0, 0, 0, 0};
        for (int i = 0; i < 4; ++i)
        {
                unsigned __int128 carry = 0;
                for (int j = 0; i + j < 4; ++j)
                {
                        const unsigned __int128 t = (unsigned __int128)a.w[i] * b.w[j] + r[i + j] + carry;
                        r[i + j] = (uint64_t)t;
                        carry = t >> 64;
                }
        }
        I256 p{{r[0], r[1], r[2], r[3]}};
        return neg ? -p : p;
}

inline int sign(const I256& a)
{
        if (negative(a))
        {
                return -1;
        }
        return (a.w[0] | a.w[1] | a.w[2] | a.w[3]) ? 1 : 0;
}

inline int sign(__int128 a)
{
        return a < 0 ? -1 : (a > 0 ? 1 : 0);
}

inline double to_double(const I256& x)
{
        const bool neg = negative(x);
        const I256 a = neg ? -x : x;
        double r = 0;
        for (int i = 3; i >= 0; --i)
        {
                r = r * 18446744073709551616.0 + (double)a.w[i];
        }
        return neg ? -r : r;
}

inline double to_double(__int128 x)
{
        return (double)x;
}

template <typename Int>
inline Int make_int(long long v)
{
        if constexpr (std::is_same_v<Int, I256>)
        {
                return i256(v);
        }
        else
        {
                return (Int)v;
        }
}

// ---- exact determinants by cofactor expansion (k <= 5)

template <typename Int, int K>
Int det(const std::array<std::array<Int, K>, K>& m)
{
        if constexpr (K == 1)
        {
                return m[0][0];
        }
        else if constexpr (K == 2)
        {
                return m[0][0] * m[1][1] - m[0][1] * m[1][0];
        }
        else
        {
                Int r = make_int<Int>(0);
                for (int c = 0; c < K; ++c)
                {
                        std::array<std::array<Int, K - 1>, K - 1> sub;
                        for (int i = 1; i < K; ++i)
                        {
                                for (int j = 0, jj = 0; j < K; ++j)
                                {
                                        if (j != c)
                                        {
                                                sub[i - 1][jj++] = m[i][j];
                                        }
                                }
                        }
                        const Int t = m[0][c] * det<Int, K - 1>(sub);
                        r = (c & 1) ? r - t : r + t;
                }
                return r;
        }
}

template <int N, typename Int>
struct Facet
{
        std::array<int, N> v;          // point indices
        std::array<Int, N> normal;     // outward
        Int d;                         // normal . v[0]
        std::array<double, N> nd;      // the plane rounded to double, for the filtered side test
        double dd = 0;
        double bound = 0;              // error bound of the double side value
        std::array<int, N> nb;         // neighbour opposite v[i]
        std::vector<int> outside;      // points assigned to this facet (they see it)
        bool alive = true;
        int mark = -1;
};

template <int N, typename Int>
class Hull
{
        const std::vector<std::array<long long, N>>& P;
        std::vector<Facet<N, Int>> F;
        std::array<long long, N> interior{};  // N+1 times an interior point (sum of the first simplex)

public:
        explicit Hull(const std::vector<std::array<long long, N>>& points) : P(points)
        {
        }

        // hyperplane through the facet's vertices, oriented away from the interior point
        void plane(Facet<N, Int>& f) const
        {
                std::array<std::array<Int, N>, N - 1> e;
                for (int i = 1; i < N; ++i)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                e[i - 1][k] = make_int<Int>(P[f.v[i]][k] - P[f.v[0]][k]);
                        }
                }
                // cofactors: the minors of the last rows over column subsets, built up one row at a
                // time (Laplace expansion along the top row, each smaller minor computed once)
                std::array<Int, 1 << N> minor, next;
                for (int c = 0; c < N; ++c)
                {
                        minor[1 << c] = e[N - 2][c];
                }
                for (int r = N - 3; r >= 0; --r)
                {
                        const int size = N - 1 - r;
                        for (int mask = 0; mask < (1 << N); ++mask)
                        {
                                if (__builtin_popcount(mask) != size)
                                {
                                        continue;
                                }
                                Int acc = make_int<Int>(0);
                                int pos = 0;
                                for (int j = 0; j < N; ++j)
                                {
                                        if (!(mask & (1 << j)))
                                        {
                                                continue;
                                        }
                                        const Int t = e[r][j] * minor[mask & ~(1 << j)];
                                        acc = (pos & 1) ? acc - t : acc + t;
                                        ++pos;
                                }
                                next[mask] = acc;
                        }
                        for (int mask = 0; mask < (1 << N); ++mask)
                        {
                                if (__builtin_popcount(mask) == size)
                                {
                                        minor[mask] = next[mask];
                                }
                        }
                }
                const int all = (1 << N) - 1;
                for (int k = 0; k < N; ++k)
                {
                        const Int c = minor[all & ~(1 << k)];
                        f.normal[k] = (k & 1) ? -c : c;
                }
                f.d = dot_point(f.normal, P[f.v[0]]);
                // interior side: normal . interior < (N + 1) d
                Int s = make_int<Int>(0);
                for (int k = 0; k < N; ++k)
                {
                        s = s + f.normal[k] * make_int<Int>(interior[k]);
                }
                const Int side = s - f.d * make_int<Int>(N + 1);
                if (sign(side) > 0)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                f.normal[k] = -f.normal[k];
                        }
                        f.d = -f.d;
                }
                // double filter: |(n . p - d) - (nd . p - dd)| <= bound for every p in [0, 2^30)^N
                double mag = 0;
                for (int k = 0; k < N; ++k)
                {
                        f.nd[k] = to_double(f.normal[k]);
                        mag += std::fabs(f.nd[k]) * 1073741824.0;
                }
                f.dd = to_double(f.d);
                mag += std::fabs(f.dd);
                f.bound = mag * (4.0 * (N + 2)) * 1.1102230246251565e-16;
        }

        static Int dot_point(const std::array<Int, N>& a, const std::array<long long, N>& p)
        {
                Int s = make_int<Int>(0);
                for (int k = 0; k < N; ++k)
                {
                        s = s + a[k] * make_int<Int>(p[k]);
                }
                return s;
        }

        bool sees(const Facet<N, Int>& f, int p) const
        {
                double a = -f.dd;
                for (int k = 0; k < N; ++k)
                {
                        a += f.nd[k] * (double)P[p][k];
                }
                if (a > f.bound)
                {
                        return true;
                }
                if (a < -f.bound)
                {
                        return false;
                }
                return sign(dot_point(f.normal, P[p]) - f.d) > 0;
        }

        // rank test for the initial simplex: the points' differences span `rank` dimensions
        bool independent(const std::vector<int>& pts) const
        {
                // exact Gaussian elimination on rational values via integer Bareiss
                const int r = (int)pts.size() - 1;
                std::vector<std::vector<Int>> m(r, std::vector<Int>(N));
                for (int i = 0; i < r; ++i)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                m[i][k] = make_int<Int>(P[pts[i + 1]][k] - P[pts[0]][k]);
                        }
                }
                // the r x N matrix has rank r iff some r x r minor is non-zero
                std::vector<int> cols(N);
                std::iota(cols.begin(), cols.end(), 0);
                std::vector<bool> pick(N, false);
                std::fill(pick.begin(), pick.begin() + r, true);
                do
                {
                        std::vector<int> c;
                        for (int k = 0; k < N; ++k)
                        {
                                if (pick[k])
                                {
                                        c.push_back(k);
                                }
                        }
                        if (sign(minor(m, c)) != 0)
                        {
                                return true;
                        }
                } while (std::prev_permutation(pick.begin(), pick.end()));
                return false;
        }

        static Int minor(const std::vector<std::vector<Int>>& m, const std::vector<int>& c)
        {
                const int r = (int)c.size();
                if (r == 1)
                {
                        return m[0][c[0]];
                }
                Int s = make_int<Int>(0);
                for (int j = 0; j < r; ++j)
                {
                        std::vector<std::vector<Int>> sub(r - 1, std::vector<Int>(N));
                        std::vector<int> cc;
                        for (int q = 0; q < r; ++q)
                        {
                                if (q != j)
                                {
                                        cc.push_back(c[q]);
                                }
                        }
                        for (int i = 1; i < r; ++i)
                        {
                                sub[i - 1] = m[i];
                        }
                        const Int t = m[0][c[j]] * minor(sub, cc);
                        s = (j & 1) ? s - t : s + t;
                }
                return s;
        }

        void run(std::vector<std::array<int, N>>* out)
        {
                const int np = (int)P.size();
                // initial simplex: the first points that keep the rank growing
                std::vector<int> simplex{0};
                for (int i = 1; i < np && (int)simplex.size() < N + 1; ++i)
                {
                        simplex.push_back(i);
                        if (!independent(simplex))
                        {
                                simplex.pop_back();
                        }
                }
                if ((int)simplex.size() < N + 1)
                {
                        throw std::runtime_error("the points do not span " + std::to_string(N) + " dimensions");
                }
                for (int s : simplex)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                interior[k] += P[s][k];
                        }
                }
                for (int i = 0; i <= N; ++i)
                {
                        Facet<N, Int> f;
                        for (int j = 0, jj = 0; j <= N; ++j)
                        {
                                if (j != i)
                                {
                                        f.v[jj++] = simplex[j];
                                }
                        }
                        plane(f);
                        F.push_back(std::move(f));
                }
                // neighbours of the simplex's facets: facet i and facet j share all vertices but
                // simplex[i] and simplex[j]
                for (int i = 0; i <= N; ++i)
                {
                        for (int q = 0; q < N; ++q)
                        {
                                const int missing = F[i].v[q];
                                int j = (int)(std::find(simplex.begin(), simplex.end(), missing) - simplex.begin());
                                F[i].nb[q] = j;
                        }
                }
                std::vector<char> in_simplex(np, 0);
                for (int s : simplex)
                {
                        in_simplex[s] = 1;
                }
                for (int p = 0; p < np; ++p)
                {
                        if (in_simplex[p])
                        {
                                continue;
                        }
                        for (int i = 0; i <= N; ++i)
                        {
                                if (sees(F[i], p))
                                {
                                        F[i].outside.push_back(p);
                                        break;
                                }
                        }
                }
                std::vector<int> owner(np, -1);
                for (size_t i = 0; i < F.size(); ++i)
                {
                        for (int p : F[i].outside)
                        {
                                owner[p] = (int)i;
                        }
                }
                // insertion in the (shuffled) point order
                std::vector<int> visible, stack;
                struct Horizon
                {
                        int vis, inv, q;  // visible facet, invisible neighbour, the visible facet's slot
                };
                std::vector<Horizon> horizon;
                std::unordered_map<std::string, std::pair<int, int>> ridges;
                for (int p = 0; p < np; ++p)
                {
                        const int start = owner[p];
                        if (start < 0 || !F[start].alive)
                        {
                                continue;  // inside the hull so far
                        }
                        // visible region by search over adjacency
                        visible.clear();
                        horizon.clear();
                        stack.assign(1, start);
                        F[start].mark = p;
                        while (!stack.empty())
                        {
                                const int f = stack.back();
                                stack.pop_back();
                                visible.push_back(f);
                                for (int q = 0; q < N; ++q)
                                {
                                        const int g = F[f].nb[q];
                                        if (F[g].mark == p)
                                        {
                                                continue;
                                        }
                                        if (sees(F[g], p))
                                        {
                                                F[g].mark = p;
                                                stack.push_back(g);
                                        }
                                        else
                                        {
                                                horizon.push_back({f, g, q});
                                        }
                                }
                        }
                        // the cone over the horizon ridges
                        ridges.clear();
                        const int first_new = (int)F.size();
                        for (const Horizon& h : horizon)
                        {
                                Facet<N, Int> nf;
                                nf.v = F[h.vis].v;
                                nf.v[h.q] = p;  // the ridge is the visible facet without v[q]
                                plane(nf);
                                nf.nb[h.q] = h.inv;
                                const int id = (int)F.size();
                                // the invisible neighbour's link across the ridge now points here
                                Facet<N, Int>& u = F[h.inv];
                                for (int q = 0; q < N; ++q)
                                {
                                        if (u.nb[q] == h.vis)
                                        {
                                                u.nb[q] = id;
                                        }
                                }
                                F.push_back(std::move(nf));
                                // links between new facets: across the ridges that contain p
                                Facet<N, Int>& cur = F[id];
                                for (int q = 0; q < N; ++q)
                                {
                                        if (q == h.q)
                                        {
                                                continue;
                                        }
                                        std::array<int, N - 1> key;
                                        for (int j = 0, jj = 0; j < N; ++j)
                                        {
                                                if (j != q)
                                                {
                                                        key[jj++] = cur.v[j];
                                                }
                                        }
                                        std::sort(key.begin(), key.end());
                                        std::string k(reinterpret_cast<const char*>(key.data()), sizeof(key));
                                        auto it = ridges.find(k);
                                        if (it == ridges.end())
                                        {
                                                ridges.emplace(std::move(k), std::make_pair(id, q));
                                        }
                                        else
                                        {
                                                cur.nb[q] = it->second.first;
                                                F[it->second.first].nb[it->second.second] = id;
                                                ridges.erase(it);
                                        }
                                }
                        }
                        // orphans: reassigned among the new facets only
                        for (int f : visible)
                        {
                                F[f].alive = false;
                                for (int o : F[f].outside)
                                {
                                        if (o == p)
                                        {
                                                continue;
                                        }
                                        owner[o] = -1;
                                        for (int g = first_new; g < (int)F.size(); ++g)
                                        {
                                                if (sees(F[g], o))
                                                {
                                                        F[g].outside.push_back(o);
                                                        owner[o] = g;
                                                        break;
                                                }
                                        }
                                }
                                std::vector<int>().swap(F[f].outside);
                        }
                }
                out->clear();
                for (const Facet<N, Int>& f : F)
                {
                        if (f.alive)
                        {
                                out->push_back(f.v);
                        }
                }
        }
};

template <int N>
void convex_hull(const float* pts, long long count, std::vector<int32_t>* facets)
{
        if (count < N + 1)
        {
                throw std::runtime_error("too few points for a hull");
        }
        // shuffle_and_convert_to_unique_integer (convex_hull.cpp:657-707)
        std::vector<int> order((size_t)count);
        std::iota(order.begin(), order.end(), 0);
        std::shuffle(order.begin(), order.end(), std::mt19937_64((unsigned long long)count));
        std::array<float, N> mn, mx;
        for (int k = 0; k < N; ++k)
        {
                mn[k] = mx[k] = pts[k];
        }
        for (long long i = 1; i < count; ++i)
        {
                for (int k = 0; k < N; ++k)
                {
                        mn[k] = std::min(mn[k], pts[i * N + k]);
                        mx[k] = std::max(mx[k], pts[i * N + k]);
                }
        }
        float max_d = mx[0] - mn[0];
        for (int k = 1; k < N; ++k)
        {
                max_d = std::max(max_d, mx[k] - mn[k]);
        }
        if (!(max_d > 0))
        {
                throw std::runtime_error("all points are equal to each other");
        }
        const long long MAXV = (1ll << 30) - 1;
        const double scale = (double)MAXV / (double)max_d;
        struct KeyHash
        {
                size_t operator()(const std::array<long long, N>& a) const
                {
                        size_t h = 1469598103934665603ull;
                        for (long long x : a)
                        {
                                h = (h ^ (size_t)x) * 1099511628211ull;
                        }
                        return h;
                }
        };
        std::unordered_set<std::array<long long, N>, KeyHash> seen((size_t)count);
        std::vector<std::array<long long, N>> ip;
        std::vector<int> map;
        ip.reserve((size_t)count);
        for (long long i = 0; i < count; ++i)
        {
                const int src = order[i];
                std::array<long long, N> v;
                for (int k = 0; k < N; ++k)
                {
                        const double x = (double)(pts[(size_t)src * N + k] - mn[k]) * scale;
                        v[k] = std::llround(x);
                        if (v[k] < 0 || v[k] > MAXV)
                        {
                                throw std::runtime_error("points preprocessing error");
                        }
                }
                if (seen.insert(v).second)
                {
                        ip.push_back(v);
                        map.push_back(src);
                }
        }
        std::vector<std::array<int, N>> out;
        if constexpr (N <= 4)
        {
                Hull<N, __int128> h(ip);
                h.run(&out);
        }
        else
        {
                Hull<N, I256> h(ip);
                h.run(&out);
        }
        facets->resize(out.size() * N);
        for (size_t f = 0; f < out.size(); ++f)
        {
                for (int k = 0; k < N; ++k)
                {
                        (*facets)[f * N + k] = map[out[f][k]];
                }
        }
}
}

extern "C" {

int nt_convex_hull(int n, const float* points, int64_t count, nt_hull** out)
{
        try
        {
                if (!points || !out || n < 3 || n > 6)
                {
                        return ntrace::report_error(NT_EINVAL, "nt_convex_hull: bad arguments");
                }
                auto h = std::make_unique<nt_hull>();
                h->n = n;
                switch (n)
                {
                case 3:
                        convex_hull<3>(points, count, &h->facets);
                        break;
                case 4:
                        convex_hull<4>(points, count, &h->facets);
                        break;
                case 5:
                        convex_hull<5>(points, count, &h->facets);
                        break;
                default:
                        convex_hull<6>(points, count, &h->facets);
                        break;
                }
                *out = h.release();
                return NT_OK;
        }
        catch (const std::bad_alloc&)
        {
                return ntrace::report_error(NT_ENOMEM, "host allocation failed");
        }
        catch (const std::exception& e)
        {
                return ntrace::report_error(NT_EDEGENERATE, std::string("convex hull: ") + e.what());
        }
}

int64_t nt_hull_facet_count(nt_hull* h)
{
        return h ? (int64_t)(h->facets.size() / h->n) : -1;
}

int nt_hull_facets(nt_hull* h, int32_t* facets)
{
        if (!h || !facets)
        {
                return ntrace::report_error(NT_EINVAL, "null argument");
        }
        std::copy(h->facets.begin(), h->facets.end(), facets);
        return NT_OK;
}

int nt_hull_destroy(nt_hull* h)
{
        delete h;
        return NT_OK;
}
}
