// Host-side geometry for scene preparation: per-facet setup and the box-versus-simplex overlap test
// used by the 2^N-tree build.  Arithmetic follows the reference's operation order so that the tree
// this library builds in float is the tree the reference's Mesh<N,float> builds:
//   dot           = a0*b0, then fma(ai, bi, acc)            (src/com/vec.h:259-266)
//   normalize     = a / sqrt(dot(a, a))                      (src/com/vec.h:281-290)
//   ortho_nn      = specialised formulas for N = 2,3,4, cofactor expansion above
//                                                            (src/geometry/core/linear_algebra.h:36-236)
// The file is compiled without floating-point contraction.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <limits>

// The overlap test is also compiled for the device (the GPU tree build): same operations, same order,
// no contraction, so the device decides every box-simplex pair as the host does.
#ifdef __CUDACC__
#define NT_HD __host__ __device__
#else
#define NT_HD
#endif

namespace ntrace
{
template <typename T>
NT_HD inline void swap_values(T& a, T& b)
{
        T t = a;
        a = b;
        b = t;
}

template <int N, typename T>
using Vec = std::array<T, N>;

template <int N, typename T>
NT_HD inline T dot(const Vec<N, T>& a, const Vec<N, T>& b)
{
        T r = a[0] * b[0];
        for (int i = 1; i < N; ++i)
        {
                r = std::fma(a[i], b[i], r);
        }
        return r;
}

template <int N, typename T>
NT_HD inline Vec<N, T> normalize(const Vec<N, T>& a)
{
        T len = std::sqrt(dot<N, T>(a, a));
        Vec<N, T> r;
        for (int i = 0; i < N; ++i)
        {
                r[i] = a[i] / len;
        }
        return r;
}

template <typename T>
NT_HD inline T smax(T a, T b)
{
        return (a < b) ? b : a;
}

template <typename T>
NT_HD inline T smin(T a, T b)
{
        return (b < a) ? b : a;
}

// Determinant of the k x k minor with rows vm and columns hm, by cofactor expansion along the first
// row (linear_algebra.h:36-97).
template <int N, typename T>
T minor_det(const std::array<Vec<N, T>, N - 1>& v, const unsigned char* vm, const unsigned char* hm, int k)
{
        if (k == 1)
        {
                return v[vm[0]][hm[0]];
        }
        if (k == 2)
        {
                return v[vm[0]][hm[0]] * v[vm[1]][hm[1]] - v[vm[0]][hm[1]] * v[vm[1]][hm[0]];
        }
        if (k == 3)
        {
                T v00 = v[vm[0]][hm[0]], v01 = v[vm[0]][hm[1]], v02 = v[vm[0]][hm[2]];
                T v10 = v[vm[1]][hm[0]], v11 = v[vm[1]][hm[1]], v12 = v[vm[1]][hm[2]];
                T v20 = v[vm[2]][hm[0]], v21 = v[vm[2]][hm[1]], v22 = v[vm[2]][hm[2]];
                T d0 = v00 * (v11 * v22 - v12 * v21);
                T d1 = v01 * (v10 * v22 - v12 * v20);
                T d2 = v02 * (v10 * v21 - v11 * v20);
                return d0 - d1 + d2;
        }
        T det = 0;
        unsigned char vs[8], hs[8];
        for (int j = 1; j < k; ++j)
        {
                vs[j - 1] = vm[j];
        }
        for (int i = 0; i < k; ++i)
        {
                T entry = v[vm[0]][hm[i]];
                for (int j = 0, c = 0; j < k; ++j)
                {
                        if (j != i)
                        {
                                hs[c++] = hm[j];
                        }
                }
                T m = minor_det<N, T>(v, vs, hs, k - 1);
                if (i & 1)
                {
                        det -= entry * m;
                }
                else
                {
                        det += entry * m;
                }
        }
        return det;
}

// Vector orthogonal to N-1 vectors (linear_algebra.h:167-236).
template <int N, typename T>
Vec<N, T> ortho_nn(const std::array<Vec<N, T>, N - 1>& v)
{
        Vec<N, T> r;
        if constexpr (N == 2)
        {
                r[0] = v[0][1];
                r[1] = -v[0][0];
        }
        else if constexpr (N == 3)
        {
                r[0] = +(v[0][1] * v[1][2] - v[0][2] * v[1][1]);
                r[1] = -(v[0][0] * v[1][2] - v[0][2] * v[1][0]);
                r[2] = +(v[0][0] * v[1][1] - v[0][1] * v[1][0]);
        }
        else if constexpr (N == 4)
        {
                r[0] = +v[0][1] * (v[1][2] * v[2][3] - v[1][3] * v[2][2]) - v[0][2] * (v[1][1] * v[2][3] - v[1][3] * v[2][1]) +
                       v[0][3] * (v[1][1] * v[2][2] - v[1][2] * v[2][1]);
                r[1] = -v[0][0] * (v[1][2] * v[2][3] - v[1][3] * v[2][2]) + v[0][2] * (v[1][0] * v[2][3] - v[1][3] * v[2][0]) -
                       v[0][3] * (v[1][0] * v[2][2] - v[1][2] * v[2][0]);
                r[2] = +v[0][0] * (v[1][1] * v[2][3] - v[1][3] * v[2][1]) - v[0][1] * (v[1][0] * v[2][3] - v[1][3] * v[2][0]) +
                       v[0][3] * (v[1][0] * v[2][1] - v[1][1] * v[2][0]);
                r[3] = -v[0][0] * (v[1][1] * v[2][2] - v[1][2] * v[2][1]) + v[0][1] * (v[1][0] * v[2][2] - v[1][2] * v[2][0]) -
                       v[0][2] * (v[1][0] * v[2][1] - v[1][1] * v[2][0]);
        }
        else
        {
                unsigned char vm[8], hm[8];
                for (int i = 0; i < N - 1; ++i)
                {
                        vm[i] = static_cast<unsigned char>(i);
                }
                for (int i = 0; i < N; ++i)
                {
                        for (int j = 0, c = 0; j < N; ++j)
                        {
                                if (j != i)
                                {
                                        hm[c++] = static_cast<unsigned char>(j);
                                }
                        }
                        T m = minor_det<N, T>(v, vm, hm, N - 1);
                        r[i] = (i & 1) ? -m : m;
                }
        }
        return r;
}

// Barycentric planes of an (N-1)-simplex in the reference's formulation
// (HyperplaneSimplexGeometry::set_data, src/painter/space/hyperplane_geometry.h:83-115): plane i
// passes through the facet opposite vertex i, is orthogonal to the simplex, and is scaled so that
// vertex i lies at distance 1.  planes[i] = (normal (N), d).
template <int N, typename T>
void reference_planes(const Vec<N, T>& simplex_normal_in, const std::array<Vec<N, T>, N>& vertices,
                      std::array<std::array<T, N + 1>, N - 1>* planes)
{
        std::array<Vec<N, T>, N - 1> vectors;
        Vec<N, T> simplex_normal = simplex_normal_in;
        for (int i = 0; i < N - 1; ++i)
        {
                for (int k = 0; k < N; ++k)
                {
                        vectors[i][k] = vertices[i][k] - vertices[N - 1][k];
                }
        }
        for (int i = 0; i < N - 1; ++i)
        {
                std::swap(simplex_normal, vectors[i]);
                Vec<N, T> pn = ortho_nn<N, T>(vectors);
                std::swap(simplex_normal, vectors[i]);
                T d = dot<N, T>(vertices[N - 1], pn);
                T distance = dot<N, T>(vertices[i], pn) - d;
                for (int k = 0; k < N; ++k)
                {
                        (*planes)[i][k] = pn[k] / distance;
                }
                (*planes)[i][N] = d / distance;
        }
}

// The same affine map solved by Gaussian elimination with partial pivoting (the method of
// src/numerical/gauss.h:58-100) in double: with E = [v0-v(N-1), ..., v(N-2)-v(N-1), normal] as
// columns, the rows of E^-1 are the barycentric plane normals.  Returns the smallest |pivot| relative
// to the largest |entry| of E (a conditioning measure; tiny means near-degenerate).
template <int N>
double gauss_planes(const Vec<N, double>& unit_normal, const std::array<Vec<N, double>, N>& vertices,
                    std::array<std::array<double, N + 1>, N - 1>* planes)
{
        double a[N][2 * N];
        double amax = 0;
        for (int r = 0; r < N; ++r)
        {
                for (int c = 0; c < N - 1; ++c)
                {
                        a[r][c] = vertices[c][r] - vertices[N - 1][r];
                }
                a[r][N - 1] = unit_normal[r];
                for (int c = 0; c < N; ++c)
                {
                        a[r][N + c] = (r == c) ? 1.0 : 0.0;
                        amax = std::max(amax, std::fabs(a[r][c]));
                }
        }
        double min_pivot = std::numeric_limits<double>::infinity();
        for (int col = 0; col < N; ++col)
        {
                int piv = col;
                for (int r = col + 1; r < N; ++r)
                {
                        if (std::fabs(a[r][col]) > std::fabs(a[piv][col]))
                        {
                                piv = r;
                        }
                }
                if (piv != col)
                {
                        for (int c = 0; c < 2 * N; ++c)
                        {
                                std::swap(a[piv][c], a[col][c]);
                        }
                }
                double p = a[col][col];
                min_pivot = std::min(min_pivot, std::fabs(p));
                if (p == 0)
                {
                        return 0;
                }
                for (int r = col + 1; r < N; ++r)
                {
                        double f = a[r][col] / p;
                        for (int c = col; c < 2 * N; ++c)
                        {
                                a[r][c] -= f * a[col][c];
                        }
                }
        }
        // back substitution: a is upper triangular; solve for the inverse columns
        double x[N][N];
        for (int c = 0; c < N; ++c)
        {
                for (int r = N - 1; r >= 0; --r)
                {
                        double s = a[r][N + c];
                        for (int k = r + 1; k < N; ++k)
                        {
                                s -= a[r][k] * x[k][c];
                        }
                        x[r][c] = s / a[r][r];
                }
        }
        for (int i = 0; i < N - 1; ++i)
        {
                double d = 0;
                for (int k = 0; k < N; ++k)
                {
                        (*planes)[i][k] = x[i][k];
                        d += x[i][k] * vertices[N - 1][k];
                }
                (*planes)[i][N] = d;
        }
        return amax > 0 ? min_pivot / amax : 0;
}

// ---------------------------------------------------------------------------------------------
// Orthogonal box (ParallelotopeOrtho, src/painter/space/parallelotope_ortho.h:197-414)

template <int N, typename T>
struct Box
{
        Vec<N, T> org, size, d1, d2;

        NT_HD static Box make(const Vec<N, T>& o, const Vec<N, T>& s)
        {
                Box b;
                for (int i = 0; i < N; ++i)
                {
                        b.org[i] = o[i];
                        b.size[i] = s[i];
                        b.d1[i] = o[i] + s[i];
                        b.d2[i] = -o[i];
                }
                return b;
        }

        NT_HD bool inside(const Vec<N, T>& p) const
        {
                for (int i = 0; i < N; ++i)
                {
                        if (!(p[i] <= d1[i]) || !(-p[i] <= d2[i]))
                        {
                                return false;
                        }
                }
                return true;
        }

        // first/second slab distances (intersect_impl)
        NT_HD bool intersect_impl(const Vec<N, T>& org_r, const Vec<N, T>& dir, T* first, T* second) const
        {
                T f_max = std::numeric_limits<T>::lowest();
                T b_min = std::numeric_limits<T>::max();
                for (int i = 0; i < N; ++i)
                {
                        T s = dir[i];
                        if (s == 0)
                        {
                                T d = org_r[i];
                                if (d - d1[i] > 0 || -d - d2[i] > 0)
                                {
                                        return false;
                                }
                                continue;
                        }
                        T d = org_r[i];
                        T alpha1 = (d1[i] - d) / s;
                        T alpha2 = (d2[i] + d) / -s;
                        if (s < 0)
                        {
                                f_max = smax(alpha1, f_max);
                                b_min = smin(alpha2, b_min);
                        }
                        else
                        {
                                b_min = smin(alpha1, b_min);
                                f_max = smax(alpha2, f_max);
                        }
                        if (b_min <= 0 || b_min < f_max)
                        {
                                return false;
                        }
                }
                *first = f_max;
                *second = b_min;
                return true;
        }

        NT_HD bool intersect(const Vec<N, T>& o, const Vec<N, T>& dir, T* t) const
        {
                T first, second;
                if (intersect_impl(o, dir, &first, &second))
                {
                        *t = (first > 0) ? first : second;
                        return true;
                }
                return false;
        }

        NT_HD Vec<N, T> vertex(int k) const
        {
                Vec<N, T> v;
                for (int i = 0; i < N; ++i)
                {
                        v[i] = (k & (1 << i)) ? org[i] + size[i] : org[i];
                }
                return v;
        }
};

// ---------------------------------------------------------------------------------------------
// Simplex data for the overlap test (HyperplaneSimplexWrapperForShapeIntersection,
// src/painter/space/hyperplane_simplex_wrapper.h, constraints from hyperplane_geometry.h:120-160)

template <int N, typename T>
struct Constraint
{
        Vec<N, T> a;
        T b;
};

template <int N, typename T>
struct SimplexShape
{
        std::array<Vec<N, T>, N> v;
        Vec<N, T> normal;
        std::array<std::array<T, N + 1>, N - 1> planes;
        std::array<Constraint<N, T>, N> c;
        Constraint<N, T> c_eq;
        Vec<N, T> min, max;

        // MeshHyperplaneSimplex ctor (mesh_hyperplane_simplex.cpp:84-94); returns false if the
        // normal is not finite
        bool init(const std::array<Vec<N, T>, N>& vertices)
        {
                v = vertices;
                std::array<Vec<N, T>, N - 1> vectors;
                for (int i = 0; i < N - 1; ++i)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                vectors[i][k] = v[i + 1][k] - v[0][k];
                        }
                }
                normal = normalize<N, T>(ortho_nn<N, T>(vectors));
                for (int k = 0; k < N; ++k)
                {
                        if (!std::isfinite(normal[k]))
                        {
                                return false;
                        }
                }
                reference_planes<N, T>(normal, v, &planes);
                min = v[0];
                max = v[0];
                for (int i = 1; i < N; ++i)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                min[k] = smin(v[i][k], min[k]);
                                max[k] = smax(v[i][k], max[k]);
                        }
                }
                if constexpr (N >= 4)
                {
                        for (int i = 0; i < N - 1; ++i)
                        {
                                Vec<N, T> pn;
                                for (int k = 0; k < N; ++k)
                                {
                                        pn[k] = planes[i][k];
                                }
                                T len = std::sqrt(dot<N, T>(pn, pn));
                                for (int k = 0; k < N; ++k)
                                {
                                        c[i].a[k] = pn[k] / len;
                                }
                                c[i].b = -planes[i][N] / len;
                        }
                        std::array<Vec<N, T>, N - 1> vs;
                        for (int i = 0; i < N - 2; ++i)
                        {
                                for (int k = 0; k < N; ++k)
                                {
                                        vs[i][k] = v[i + 1][k] - v[0][k];
                                }
                        }
                        vs[N - 2] = normal;
                        Vec<N, T> nn = normalize<N, T>(ortho_nn<N, T>(vs));
                        T d = dot<N, T>(v[0], nn);
                        bool to_vertex = dot<N, T>(v[N - 1], nn) - d >= 0;
                        for (int k = 0; k < N; ++k)
                        {
                                c[N - 1].a[k] = to_vertex ? nn[k] : -nn[k];
                        }
                        c[N - 1].b = to_vertex ? -d : d;
                        d = dot<N, T>(v[0], normal);
                        c_eq.a = normal;
                        c_eq.b = -d;
                }
                return true;
        }

        // HyperplaneSimplexGeometry::intersect with the ray direction normalised from `direction`
        NT_HD bool intersect(const Vec<N, T>& org, const Vec<N, T>& dir, T* t) const
        {
                T s = dot<N, T>(normal, dir);
                if (!(s != 0))
                {
                        return false;
                }
                Vec<N, T> diff;
                for (int k = 0; k < N; ++k)
                {
                        diff[k] = v[0][k] - org[k];
                }
                *t = dot<N, T>(diff, normal) / s;
                if (!(*t > 0))
                {
                        return false;
                }
                Vec<N, T> p;
                for (int k = 0; k < N; ++k)
                {
                        p[k] = org[k] + dir[k] * *t;
                }
                T coords[N];
                for (int i = 0; i < N - 1; ++i)
                {
                        Vec<N, T> pn;
                        for (int k = 0; k < N; ++k)
                        {
                                pn[k] = planes[i][k];
                        }
                        coords[i] = dot<N, T>(p, pn) - planes[i][N];
                        if (coords[i] <= 0 || coords[i] >= 1)
                        {
                                return false;
                        }
                }
                T r = 1;
                for (int i = 0; i < N - 1; ++i)
                {
                        r -= coords[i];
                }
                return r > 0;
        }
};

// CLRS simplex-method feasibility test of a x + b >= 0 (src/numerical/simplex.h:160-441).
template <int NS, typename T, int M>
NT_HD bool lp_feasible(const std::array<Vec<NS, T>, M>& a_in, const std::array<T, M>& b_in)
{
        constexpr int N = NS + 1;
        long long max_iter = 1;
        for (int i = 1; i <= M; ++i)
        {
                max_iter = max_iter * (N + i) / i;
        }
        std::array<T, M> b = b_in;
        T mn = b[0];
        for (int m = 1; m < M; ++m)
        {
                mn = smin(b[m], mn);
        }
        if (mn >= 0)
        {
                return true;
        }
        T a[M][N];
        T c[N];
        T v = 0;
        int map_n[N], map_m[M];
        for (int m = 0; m < M; ++m)
        {
                T mx = std::fabs(a_in[m][0]);
                for (int k = 1; k < NS; ++k)
                {
                        mx = smax(mx, std::fabs(a_in[m][k]));
                }
                mx = (mx != 0) ? mx : 1;
                T rec = 1 / mx;
                b[m] *= rec;
                a[m][0] = 1;
                for (int k = 0; k < NS; ++k)
                {
                        a[m][k + 1] = a_in[m][k] * rec;
                }
        }
        c[0] = -1;
        for (int k = 1; k < N; ++k)
        {
                c[k] = 0;
        }
        for (int i = 0; i < N; ++i)
        {
                map_n[i] = i;
        }
        for (int i = 0; i < M; ++i)
        {
                map_m[i] = i + N;
        }
        auto pivot = [&](int l, int e) {
                b[l] = -b[l] / a[l][e];
                for (int j = 0; j < N; ++j)
                {
                        if (j != e)
                        {
                                a[l][j] = -a[l][j] / a[l][e];
                        }
                }
                a[l][e] = 1 / a[l][e];
                for (int i = 0; i < M; ++i)
                {
                        if (i == l)
                        {
                                continue;
                        }
                        b[i] = b[i] + a[i][e] * b[l];
                        for (int j = 0; j < N; ++j)
                        {
                                if (j != e)
                                {
                                        a[i][j] = a[i][j] + a[i][e] * a[l][j];
                                }
                        }
                        a[i][e] = a[i][e] * a[l][e];
                }
                v = v + c[e] * b[l];
                for (int j = 0; j < N; ++j)
                {
                        if (j != e)
                        {
                                c[j] = c[j] + c[e] * a[l][j];
                        }
                }
                c[e] = c[e] * a[l][e];
        };
        mn = b[0];
        int k = 0;
        for (int m = 1; m < M; ++m)
        {
                if (b[m] < mn)
                {
                        mn = b[m];
                        k = m;
                }
        }
        if (mn >= 0)
        {
                return true;
        }
        pivot(k, 0);
        swap_values(map_m[k], map_n[0]);
        for (long long iteration = 2;; ++iteration)
        {
                T max_abs_c = std::fabs(c[0]);
                for (int i = 1; i < N; ++i)
                {
                        max_abs_c = smax(max_abs_c, std::fabs(c[i]));
                }
                T eps_c = max_abs_c * (2 * std::numeric_limits<T>::epsilon());
                int e = -1;
                for (int i = 0; i < N; ++i)
                {
                        if (c[i] > eps_c)
                        {
                                e = i;
                                break;
                        }
                }
                if (e < 0)
                {
                        break;
                }
                if (iteration >= max_iter)
                {
                        return false;
                }
                T max_delta = std::numeric_limits<T>::lowest();
                int l = -1;
                for (int i = 0; i < M; ++i)
                {
                        b[i] = (0 < b[i]) ? b[i] : T(0);
                        if (a[i][e] < 0)
                        {
                                T delta = b[i] / a[i][e];
                                if (delta > max_delta || l < 0)
                                {
                                        max_delta = delta;
                                        l = i;
                                }
                        }
                }
                if (l < 0)
                {
                        return false;
                }
                pivot(l, e);
                swap_values(map_m[l], map_n[e]);
        }
        for (int i = 0; i < N; ++i)
        {
                if (map_n[i] == 0)
                {
                        return true;
                }
        }
        for (int i = 0; i < M; ++i)
        {
                if (map_m[i] == 0 && b[i] <= 0)
                {
                        return true;
                }
        }
        return false;
}

// shape_intersection(box, simplex, 10 epsilons) (src/painter/space/shape_intersection.h:343-385)
template <int N, typename T>
NT_HD bool box_simplex_overlap(const Box<N, T>& box, const SimplexShape<N, T>& s)
{
        constexpr int VC = 1 << N;
        for (int i = 0; i < N; ++i)
        {
                if (box.inside(s.v[i]))
                {
                        return true;
                }
        }
        if constexpr (N <= 3)
        {
                auto seg_hits_simplex = [&](const Vec<N, T>& org, const Vec<N, T>& direction) {
                        Vec<N, T> dir = normalize<N, T>(direction);
                        T alpha;
                        return s.intersect(org, dir, &alpha) && (alpha * alpha < dot<N, T>(direction, direction));
                };
                auto seg_hits_box = [&](const Vec<N, T>& org, const Vec<N, T>& direction) {
                        Vec<N, T> dir = normalize<N, T>(direction);
                        T alpha;
                        return box.intersect(org, dir, &alpha) && (alpha * alpha < dot<N, T>(direction, direction));
                };
                for (int k = 0; k < VC; ++k)
                {
                        Vec<N, T> v = box.vertex(k);
                        for (int i = 0; i < N; ++i)
                        {
                                if (k & (1 << i))
                                {
                                        continue;
                                }
                                Vec<N, T> e{};
                                e[i] = box.size[i];
                                if (seg_hits_simplex(v, e))
                                {
                                        return true;
                                }
                        }
                }
                for (int i = 0; i < N - 1; ++i)
                {
                        for (int j = i + 1; j < N; ++j)
                        {
                                Vec<N, T> d;
                                for (int k = 0; k < N; ++k)
                                {
                                        d[k] = s.v[j][k] - s.v[i][k];
                                }
                                if (seg_hits_box(s.v[i], d))
                                {
                                        return true;
                                }
                        }
                }
                return false;
        }
        else
        {
                // shapes_not_intersect_by_planes
                std::array<Constraint<N, T>, 2 * N> bc;
                for (int i = 0; i < N; ++i)
                {
                        for (int k = 0; k < N; ++k)
                        {
                                bc[2 * i].a[k] = (k == i) ? T(-1) : T(0);
                                bc[2 * i + 1].a[k] = (k == i) ? T(1) : T(0);
                        }
                        bc[2 * i].b = box.d1[i];
                        bc[2 * i + 1].b = box.d2[i];
                }
                for (const auto& c : bc)
                {
                        bool all_negative = true;
                        for (int i = 0; i < N; ++i)
                        {
                                if (dot<N, T>(s.v[i], c.a) + c.b > 0)
                                {
                                        all_negative = false;
                                        break;
                                }
                        }
                        if (all_negative)
                        {
                                return false;
                        }
                }
                std::array<Vec<N, T>, VC> bv;
                for (int k = 0; k < VC; ++k)
                {
                        bv[k] = box.vertex(k);
                }
                for (int q = 0; q < N; ++q)
                {
                        bool all_negative = true;
                        for (int k = 0; k < VC; ++k)
                        {
                                if (dot<N, T>(bv[k], s.c[q].a) + s.c[q].b > 0)
                                {
                                        all_negative = false;
                                        break;
                                }
                        }
                        if (all_negative)
                        {
                                return false;
                        }
                }
                {
                        // all_vertices_are_on_the_same_side compares each vertex with the previous one
                        bool negative = false, positive = false, same = true;
                        for (int k = 0; k < VC; ++k)
                        {
                                T p = dot<N, T>(bv[k], s.c_eq.a) + s.c_eq.b;
                                if ((p > 0 && negative) || (p < 0 && positive))
                                {
                                        same = false;
                                        break;
                                }
                                negative = p < 0;
                                positive = p > 0;
                        }
                        if (same)
                        {
                                return false;
                        }
                }
                // shapes_intersect_by_spaces
                Vec<N, T> mn;
                T max_value = 0;
                for (int k = 0; k < N; ++k)
                {
                        mn[k] = smin(box.org[k], s.min[k]);
                }
                for (int k = 0; k < N; ++k)
                {
                        T d = smax(box.org[k] + box.size[k], s.max[k]) - mn[k];
                        max_value = (k == 0) ? d : smax(max_value, d);
                }
                const T distance = max_value * (T(10) * std::numeric_limits<T>::epsilon());
                constexpr int M = 3 * N + 2;
                std::array<Vec<N, T>, M> a;
                std::array<T, M> b;
                int i = 0;
                for (const auto& c : bc)
                {
                        a[i] = c.a;
                        b[i] = dot<N, T>(c.a, mn) + c.b;
                        ++i;
                }
                for (const auto& c : s.c)
                {
                        a[i] = c.a;
                        b[i] = dot<N, T>(c.a, mn) + c.b;
                        ++i;
                }
                T b_v = dot<N, T>(s.c_eq.a, mn) + s.c_eq.b;
                a[i] = s.c_eq.a;
                b[i] = b_v + distance;
                ++i;
                for (int k = 0; k < N; ++k)
                {
                        a[i][k] = -s.c_eq.a[k];
                }
                b[i] = -b_v + distance;
                return lp_feasible<N, T, M>(a, b);
        }
}
}
