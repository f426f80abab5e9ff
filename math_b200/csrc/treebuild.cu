// 2^N-tree build on the GPU (treebuild.h).
//
// Level by level, as the host build: the boxes of a level that hold more than min_objects facets (and
// are above the depth limit) split into 2^N children with contiguous node numbers in parent order.
// For every child, one block tests the parent's facets against the child box (box_simplex_overlap,
// the host's code compiled for the device) and records the outcomes as a bit mask (warp ballots) and
// a count; after a prefix sum of the counts on the host, one warp per child writes the facets that
// overlap, in the parent's list order.  Leaves keep their level's list; the leaf index array is their
// lists in node order (breadth-first numbering makes level order node order).
#include "treebuild.h"

#include <algorithm>
#include <memory>

namespace ntrace
{
namespace
{
constexpr int TB = 256;

template <int N>
struct ChildDesc
{
        Vec<N, float> org;
        long long list_off;   // parent's list in the current level's buffer
        long long list_cnt;
        long long word_off;   // this child's segment of the bit masks
};

template <int N>
__global__ void __launch_bounds__(TB) k_overlap(const SimplexShape<N, float>* __restrict__ shapes,
                                                const int* __restrict__ list_cur, const ChildDesc<N>* __restrict__ kids,
                                                long long nkids, Vec<N, float> half, unsigned* __restrict__ bits,
                                                unsigned* __restrict__ counts, unsigned long long* tests)
{
        __shared__ unsigned s_count;
        const int lane = threadIdx.x & 31;
        const int warp = threadIdx.x >> 5;
        for (long long c = blockIdx.x; c < nkids; c += gridDim.x)
        {
                const ChildDesc<N> d = kids[c];
                const Box<N, float> box = Box<N, float>::make(d.org, half);
                if (threadIdx.x == 0)
                {
                        s_count = 0;
                }
                __syncthreads();
                unsigned mine = 0;
                for (long long j0 = 0; j0 < d.list_cnt; j0 += TB)
                {
                        const long long j = j0 + threadIdx.x;
                        bool hit = false;
                        if (j < d.list_cnt)
                        {
                                hit = box_simplex_overlap<N, float>(box, shapes[list_cur[d.list_off + j]]);
                        }
                        const unsigned b = __ballot_sync(0xffffffffu, hit);
                        if (lane == 0 && j0 + warp * 32 < d.list_cnt)
                        {
                                bits[d.word_off + (j0 >> 5) + warp] = b;
                                mine += __popc(b);
                        }
                }
                if (lane == 0)
                {
                        atomicAdd(&s_count, mine);
                }
                __syncthreads();
                if (threadIdx.x == 0)
                {
                        counts[c] = s_count;
                        atomicAdd(tests, (unsigned long long)d.list_cnt);
                }
                __syncthreads();
        }
}

template <int N>
__global__ void __launch_bounds__(TB) k_write(const int* __restrict__ list_cur, const ChildDesc<N>* __restrict__ kids,
                                              long long nkids, const unsigned* __restrict__ bits,
                                              const long long* __restrict__ out_off, int* __restrict__ list_next)
{
        const int lane = threadIdx.x & 31;
        const long long warps = (long long)gridDim.x * (TB / 32);
        unsigned lt;
        asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
        for (long long c = (long long)blockIdx.x * (TB / 32) + (threadIdx.x >> 5); c < nkids; c += warps)
        {
                const ChildDesc<N> d = kids[c];
                const long long words = (d.list_cnt + 31) >> 5;
                long long pos = out_off[c];
                for (long long w = 0; w < words; ++w)
                {
                        const unsigned b = bits[d.word_off + w];
                        if ((b >> lane) & 1u)
                        {
                                list_next[pos + __popc(b & lt)] = list_cur[d.list_off + w * 32 + lane];
                        }
                        pos += __popc(b);
                }
        }
}

struct Dev
{
        void* p = nullptr;
        ~Dev()
        {
                if (p)
                {
                        cudaFree(p);
                }
        }
        cudaError_t alloc(size_t bytes)
        {
                if (p)
                {
                        cudaFree(p);
                        p = nullptr;
                }
                return cudaMalloc(&p, std::max<size_t>(bytes, 16));
        }
};

#define TB_CHECK(call, what)                                                  \
        do                                                                    \
        {                                                                     \
                cudaError_t e_ = (call);                                      \
                if (e_ != cudaSuccess)                                        \
                {                                                             \
                        out->error = e_;                                      \
                        out->message = std::string(what) + ": " + cudaGetErrorString(e_); \
                        return;                                               \
                }                                                             \
        } while (0)
}

template <int N>
void build_tree_gpu(const std::vector<SimplexShape<N, float>>& shapes, const Vec<N, float>& root_org,
                    const std::vector<float>& level_sizes, int max_depth, int min_objects, cudaStream_t st,
                    TreeResult* out)
{
        const long long nf = (long long)shapes.size();
        constexpr int C = 1 << N;
        Dev d_shapes, d_tests;
        TB_CHECK(d_shapes.alloc(sizeof(SimplexShape<N, float>) * (size_t)nf), "cudaMalloc");
        TB_CHECK(cudaMemcpyAsync(d_shapes.p, shapes.data(), sizeof(SimplexShape<N, float>) * (size_t)nf,
                                 cudaMemcpyHostToDevice, st),
                 "upload");
        TB_CHECK(d_tests.alloc(sizeof(unsigned long long)), "cudaMalloc");
        TB_CHECK(cudaMemsetAsync(d_tests.p, 0, sizeof(unsigned long long), st), "memset");

        // one list buffer per level (leaves keep pointing into theirs)
        std::vector<std::unique_ptr<Dev>> lists;
        std::vector<long long> list_sizes;
        {
                std::vector<int> all((size_t)nf);
                for (long long f = 0; f < nf; ++f)
                {
                        all[f] = (int)f;
                }
                lists.push_back(std::make_unique<Dev>());
                TB_CHECK(lists.back()->alloc(sizeof(int) * (size_t)nf), "cudaMalloc");
                TB_CHECK(cudaMemcpyAsync(lists.back()->p, all.data(), sizeof(int) * (size_t)nf, cudaMemcpyHostToDevice, st),
                         "upload");
                TB_CHECK(cudaStreamSynchronize(st), "sync");
                list_sizes.push_back(nf);
        }
        struct BoxRef
        {
                long long node;
                Vec<N, float> org;
                long long off, cnt;
        };
        struct LeafRef
        {
                long long node;
                int level;
                long long off, cnt;
        };
        std::vector<BoxRef> cur(1);
        cur[0] = {0, root_org, 0, nf};
        std::vector<LeafRef> leaves;
        std::vector<int32_t> nodes(2, 0);
        long long node_count = 1;
        for (int depth = 1; !cur.empty(); ++depth)
        {
                const int level = depth - 1;  // the list buffer of `cur`
                std::vector<long long> split;
                for (long long i = 0; i < (long long)cur.size(); ++i)
                {
                        if (depth >= max_depth || cur[i].cnt <= min_objects)
                        {
                                leaves.push_back({cur[i].node, level, cur[i].off, cur[i].cnt});
                        }
                        else
                        {
                                split.push_back(i);
                        }
                }
                if (split.empty())
                {
                        break;
                }
                const long long nkids = (long long)split.size() * C;
                nodes.resize((size_t)(node_count + nkids) * 2, 0);
                std::vector<ChildDesc<N>> kids((size_t)nkids);
                Vec<N, float> half;
                for (int k = 0; k < N; ++k)
                {
                        half[k] = level_sizes[(size_t)depth * N + k];
                }
                long long words = 0;
                for (size_t s = 0; s < split.size(); ++s)
                {
                        const BoxRef& parent = cur[split[s]];
                        const long long first = node_count + (long long)s * C;
                        nodes[parent.node * 2 + 0] = (int32_t)first;
                        nodes[parent.node * 2 + 1] = -1;
                        for (int c = 0; c < C; ++c)
                        {
                                ChildDesc<N>& d = kids[s * C + c];
                                for (int k = 0; k < N; ++k)
                                {
                                        const float org_plus_half = parent.org[k] + half[k];
                                        d.org[k] = (c & (1 << k)) ? org_plus_half : parent.org[k];
                                }
                                d.list_off = parent.off;
                                d.list_cnt = parent.cnt;
                                d.word_off = words;
                                words += (parent.cnt + 31) / 32;
                        }
                }
                Dev d_kids, d_bits, d_counts, d_off;
                TB_CHECK(d_kids.alloc(sizeof(ChildDesc<N>) * (size_t)nkids), "cudaMalloc");
                TB_CHECK(d_bits.alloc(sizeof(unsigned) * (size_t)words), "cudaMalloc");
                TB_CHECK(d_counts.alloc(sizeof(unsigned) * (size_t)nkids), "cudaMalloc");
                TB_CHECK(cudaMemcpyAsync(d_kids.p, kids.data(), sizeof(ChildDesc<N>) * (size_t)nkids, cudaMemcpyHostToDevice,
                                         st),
                         "upload");
                const unsigned grid = (unsigned)std::min<long long>(nkids, 148LL * 64);
                k_overlap<N><<<grid, TB, 0, st>>>(static_cast<const SimplexShape<N, float>*>(d_shapes.p),
                                                  static_cast<const int*>(lists[level]->p),
                                                  static_cast<const ChildDesc<N>*>(d_kids.p), nkids, half,
                                                  static_cast<unsigned*>(d_bits.p), static_cast<unsigned*>(d_counts.p),
                                                  static_cast<unsigned long long*>(d_tests.p));
                TB_CHECK(cudaGetLastError(), "overlap kernel");
                std::vector<unsigned> counts((size_t)nkids);
                TB_CHECK(cudaMemcpyAsync(counts.data(), d_counts.p, sizeof(unsigned) * (size_t)nkids, cudaMemcpyDeviceToHost,
                                         st),
                         "copy");
                TB_CHECK(cudaStreamSynchronize(st), "overlap");
                std::vector<long long> off((size_t)nkids);
                long long total = 0;
                for (long long c = 0; c < nkids; ++c)
                {
                        off[c] = total;
                        total += counts[c];
                }
                TB_CHECK(d_off.alloc(sizeof(long long) * (size_t)nkids), "cudaMalloc");
                TB_CHECK(cudaMemcpyAsync(d_off.p, off.data(), sizeof(long long) * (size_t)nkids, cudaMemcpyHostToDevice, st),
                         "upload");
                lists.push_back(std::make_unique<Dev>());
                TB_CHECK(lists.back()->alloc(sizeof(int) * (size_t)total), "cudaMalloc");
                list_sizes.push_back(total);
                const unsigned wgrid = (unsigned)std::min<long long>((nkids + TB / 32 - 1) / (TB / 32), 148LL * 64);
                k_write<N><<<wgrid, TB, 0, st>>>(static_cast<const int*>(lists[level]->p),
                                                 static_cast<const ChildDesc<N>*>(d_kids.p), nkids,
                                                 static_cast<const unsigned*>(d_bits.p),
                                                 static_cast<const long long*>(d_off.p), static_cast<int*>(lists.back()->p));
                TB_CHECK(cudaGetLastError(), "write kernel");
                TB_CHECK(cudaStreamSynchronize(st), "write");
                std::vector<BoxRef> next((size_t)nkids);
                for (long long c = 0; c < nkids; ++c)
                {
                        next[c] = {node_count + c, kids[c].org, off[c], (long long)counts[c]};
                }
                node_count += nkids;
                if (node_count > (1ll << 31) - 1)
                {
                        out->error = cudaErrorInvalidValue;
                        out->message = "tree too large";
                        return;
                }
                cur.swap(next);
        }
        // leaf lists in node order (levels are in node order, and so are the boxes within a level)
        std::sort(leaves.begin(), leaves.end(), [](const LeafRef& a, const LeafRef& b) { return a.node < b.node; });
        std::vector<std::vector<int>> host_lists(lists.size());
        for (size_t l = 0; l < lists.size(); ++l)
        {
                host_lists[l].resize((size_t)list_sizes[l]);
                if (list_sizes[l] > 0)
                {
                        TB_CHECK(cudaMemcpyAsync(host_lists[l].data(), lists[l]->p, sizeof(int) * (size_t)list_sizes[l],
                                                 cudaMemcpyDeviceToHost, st),
                                 "copy");
                }
        }
        unsigned long long tests = 0;
        TB_CHECK(cudaMemcpyAsync(&tests, d_tests.p, sizeof(tests), cudaMemcpyDeviceToHost, st), "copy");
        TB_CHECK(cudaStreamSynchronize(st), "sync");
        out->leaf_idx.clear();
        for (const LeafRef& lf : leaves)
        {
                nodes[lf.node * 2 + 0] = (int32_t)out->leaf_idx.size();
                nodes[lf.node * 2 + 1] = (int32_t)lf.cnt;
                const std::vector<int>& src = host_lists[lf.level];
                out->leaf_idx.insert(out->leaf_idx.end(), src.begin() + lf.off, src.begin() + lf.off + lf.cnt);
        }
        if (out->leaf_idx.empty())
        {
                out->leaf_idx.push_back(0);
        }
        out->nodes.swap(nodes);
        out->leaf_count = (long long)leaves.size();
        out->overlap_tests = (long long)tests;
}

#define NT_TREE_INSTANTIATE(N)                                                                                    \
        template void build_tree_gpu<N>(const std::vector<SimplexShape<N, float>>&, const Vec<N, float>&,          \
                                        const std::vector<float>&, int, int, cudaStream_t, TreeResult*);
NT_TREE_INSTANTIATE(3)
NT_TREE_INSTANTIATE(4)
NT_TREE_INSTANTIATE(5)
NT_TREE_INSTANTIATE(6)
#undef NT_TREE_INSTANTIATE
}
