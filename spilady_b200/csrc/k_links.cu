// links(): link-cell membership and the per-cell member lists.
//
// The reference keeps a doubly linked list per cell (links_CPU.cpp:33-177):
// atoms are first pushed at the head in index order, and every step the
// atoms whose cell changed are unlinked and pushed at the head of their new
// cell in ascending atom index.  So the head -> tail order of a cell is the
// order of descending "insertion time".  Here every atom carries that time as
// a 64-bit stamp (initial insertion: its index; a move in links call L:
// L * 2^32 + index) and the lists are rebuilt in parallel each step:
// count -> scan -> scatter -> per-cell sort by descending stamp.  The result
// is the reference's list order exactly, with no serial relink.
#include "sld_common.cuh"

__global__ void k_zero_counts(Dev D) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < D.ncells) D.cell_count[c] = 0;
    if (D.te_mesh > 0 && c < D.nte) D.te_count[c] = 0;
}

// atomicAdd(&a[key], 1) for every lane with key >= 0, one atomic per
// distinct key of the warp (the leader adds the count of its peers): the
// atoms of a warp mostly share a few link cells and one Te node.  Returns
// this lane's rank among its peers.  All 32 lanes must call it.
__device__ __forceinline__ int warp_count_add(int* a, int key, int* base_out) {
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (key >= 0 && lane == leader) base = atomicAdd(a + key, __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (base_out) *base_out = base;
    return __popc(peers & ((1u << lane) - 1u));
}

__global__ void k_bin(Dev D, int initial) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < D.natom;
    int c = -1, k = -1;
    if (valid) {
        double4 r = D.r[i];
        double3 q = to_frac(D, r.x, r.y, r.z);
        int lx = (int)(q.x * D.nx), ly = (int)(q.y * D.ny), lz = (int)(q.z * D.nz);
        lx = lx < 0 ? 0 : (lx >= D.nx ? D.nx - 1 : lx);
        ly = ly < 0 ? 0 : (ly >= D.ny ? D.ny - 1 : ly);
        lz = lz < 0 ? 0 : (lz >= D.nz ? D.nz - 1 : lz);
        c = lx + (ly + lz * D.ny) * D.nx;
        int id = D.id[i];
        if (initial) {
            D.stamp[i] = (long long)id;
        } else if (c != D.cell_of[i]) {
            long long L = D.ctl->links_calls + 1;
            D.stamp[i] = (L << 32) | (long long)id;
        }
        D.cell_of[i] = c;
        if (D.te_mesh > 0) {
            int a = (int)(q.x * D.tx), b = (int)(q.y * D.ty), e = (int)(q.z * D.tz);
            a = a < 0 ? 0 : (a >= D.tx ? D.tx - 1 : a);
            b = b < 0 ? 0 : (b >= D.ty ? D.ty - 1 : b);
            e = e < 0 ? 0 : (e >= D.tz ? D.tz - 1 : e);
            k = a + (b + e * D.ty) * D.tx;
            D.node[i] = k;
        }
    }
    warp_count_add(D.cell_count, c, nullptr);
    if (D.te_mesh > 0) warp_count_add(D.te_count, k, nullptr);
}

// inclusive warp scan
__device__ __forceinline__ int warp_iscan(int v) {
    int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// exclusive scan of 1024 values per block; returns the exclusive prefix,
// block total in *total
__device__ __forceinline__ int block_escan(int v, int* total) {
    __shared__ int ws[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = warp_iscan(v);
    if (lane == 31) ws[w] = inc;
    __syncthreads();
    if (w == 0) {
        int t = ws[lane];
        t = warp_iscan(t);
        ws[lane] = t;
    }
    __syncthreads();
    int base = w > 0 ? ws[w - 1] : 0;
    *total = ws[31];
    __syncthreads();
    return base + inc - v;
}

__global__ void __launch_bounds__(1024) k_scan1(Dev D) {
    int c = blockIdx.x * 1024 + threadIdx.x;
    int v = c < D.ncells ? D.cell_count[c] : 0;
    int tot;
    int ex = block_escan(v, &tot);
    if (c < D.ncells) D.cell_start[c] = ex;
    if (threadIdx.x == 0) D.scan_tmp[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) k_scan2(Dev D, int nblocks, int bump) {
    int carry = 0;
    for (int base = 0; base < nblocks; base += 1024) {
        int b = base + threadIdx.x;
        int v = b < nblocks ? D.scan_tmp[b] : 0;
        int tot;
        int ex = block_escan(v, &tot);
        if (b < nblocks) D.scan_tmp[b] = ex + carry;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0 && bump) D.ctl->links_calls += 1;
}

__global__ void __launch_bounds__(1024) k_scan3(Dev D) {
    int c = blockIdx.x * 1024 + threadIdx.x;
    if (c < D.ncells) {
        D.cell_start[c] += D.scan_tmp[blockIdx.x];
        D.cell_fill[c] = 0;
    }
}

__global__ void k_scatter(Dev D) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = i < D.natom ? D.cell_of[i] : -1;
    int base = 0;
    const int rank = warp_count_add(D.cell_fill, c, &base);
    if (c >= 0) D.cell_atoms[D.cell_start[c] + base + rank] = i;
}

// Order each cell's members by descending stamp (head first), then record
// each member's slot and its FP32 position in slot order.
__global__ void k_cellsort(Dev D) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= D.ncells) return;
    int st = D.cell_start[c];
    if (D.cell_count[c] > SLD_MAXC) atomicOr(&D.ctl->err, SLD_FLAG_CAPACITY);
    const int n = cell_n(D, c);
    int* a = D.cell_atoms + st;
    for (int k = 1; k < n; ++k) {
        int v = a[k];
        long long key = D.stamp[v];
        int m = k - 1;
        while (m >= 0 && D.stamp[a[m]] < key) {
            a[m + 1] = a[m];
            --m;
        }
        a[m + 1] = v;
    }
    for (int k = 0; k < n; ++k) {
        int i = a[k];
        D.cell_slot[i] = st + k;
        double4 r = D.r[i];
        const int4 q = cell_fix(D, c, r.x, r.y, r.z);
        D.fxs[st + k] = q;
        if (D.fxa) D.fxa[i] = q;
    }
}

void launch_links(const Dev& D, cudaStream_t st, bool initial, int scan_blocks) {
    int big = D.ncells > D.nte ? D.ncells : D.nte;
    k_zero_counts<<<div_up(big, 256), 256, 0, st>>>(D);
    k_bin<<<div_up(D.natom, 256), 256, 0, st>>>(D, initial ? 1 : 0);
    k_scan1<<<scan_blocks, 1024, 0, st>>>(D);
    k_scan2<<<1, 1024, 0, st>>>(D, scan_blocks, initial ? 0 : 1);
    k_scan3<<<scan_blocks, 1024, 0, st>>>(D);
    k_scatter<<<div_up(D.natom, 256), 256, 0, st>>>(D);
    k_cellsort<<<div_up(D.ncells, 128), 128, 0, st>>>(D);
}
