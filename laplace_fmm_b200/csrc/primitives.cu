// Exclusive scan and stable LSD radix sort (see primitives.cuh).
#include "primitives.cuh"

namespace lfmm {

namespace {

constexpr int SCAN_BLOCK = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

// Block-wide exclusive scan of one value per thread; returns the block total.
template <int BLOCK>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t& excl, uint32_t* warp_tot)
{
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	uint32_t inc = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
		if (lane >= o) inc += t;
	}
	if (lane == 31) warp_tot[warp] = inc;
	__syncthreads();
	if (warp == 0) {
		constexpr int NW = BLOCK / 32;
		uint32_t w = lane < NW ? warp_tot[lane] : 0u;
		uint32_t wi = w;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
			if (lane >= o) wi += t;
		}
		if (lane < NW) warp_tot[lane] = wi - w;     // exclusive warp offsets
		if (lane == 31) warp_tot[32] = wi;          // block total
	}
	__syncthreads();
	excl = inc - v + warp_tot[warp];
	uint32_t total = warp_tot[32];
	__syncthreads();
	return total;
}

__global__ void __launch_bounds__(SCAN_BLOCK) scan_reduce_kernel(const uint32_t* __restrict__ in, size_t n,
                                                                 uint32_t* __restrict__ sums)
{
	__shared__ uint32_t warp_tot[33];
	size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
	uint32_t s = 0;
#pragma unroll
	for (int i = 0; i < SCAN_ITEMS; ++i)
		if (base + i < n) s += in[base + i];
	uint32_t excl;
	uint32_t tot = block_exclusive_scan<SCAN_BLOCK>(s, excl, warp_tot);
	if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Single block: exclusive scan of the block sums in place, total to *total.
__global__ void __launch_bounds__(SCAN_BLOCK) scan_sums_kernel(uint32_t* sums, size_t nb, uint32_t* total)
{
	__shared__ uint32_t warp_tot[33];
	uint32_t carry = 0;
	for (size_t start = 0; start < nb; start += SCAN_TILE) {
		size_t base = start + (size_t)threadIdx.x * SCAN_ITEMS;
		uint32_t v[SCAN_ITEMS];
		uint32_t s = 0;
#pragma unroll
		for (int i = 0; i < SCAN_ITEMS; ++i) { v[i] = base + i < nb ? sums[base + i] : 0u; s += v[i]; }
		uint32_t excl;
		uint32_t tot = block_exclusive_scan<SCAN_BLOCK>(s, excl, warp_tot);
		uint32_t run = carry + excl;
#pragma unroll
		for (int i = 0; i < SCAN_ITEMS; ++i) {
			if (base + i < nb) sums[base + i] = run;
			run += v[i];
		}
		carry += tot;
	}
	if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void __launch_bounds__(SCAN_BLOCK) scan_apply_kernel(const uint32_t* in, uint32_t* out, size_t n,
                                                                const uint32_t* __restrict__ sums)
{
	__shared__ uint32_t warp_tot[33];
	size_t base = (size_t)blockIdx.x * SCAN_TILE + (size_t)threadIdx.x * SCAN_ITEMS;
	uint32_t v[SCAN_ITEMS];
	uint32_t s = 0;
#pragma unroll
	for (int i = 0; i < SCAN_ITEMS; ++i) { v[i] = base + i < n ? in[base + i] : 0u; s += v[i]; }
	uint32_t excl;
	block_exclusive_scan<SCAN_BLOCK>(s, excl, warp_tot);
	uint32_t run = sums[blockIdx.x] + excl;
#pragma unroll
	for (int i = 0; i < SCAN_ITEMS; ++i) {
		if (base + i < n) out[base + i] = run;
		run += v[i];
	}
}

// ---------------------------------------------------------------- radix
constexpr int RADIX_BLOCK = 256;
constexpr int RADIX_ROUNDS = 16;
constexpr int RADIX_TILE = RADIX_BLOCK * RADIX_ROUNDS;   // 4096 keys per tile
constexpr int RADIX_DIGITS = 256;

__global__ void __launch_bounds__(RADIX_BLOCK) radix_hist_kernel(const uint64_t* __restrict__ keys, size_t n, int shift,
                                                                 uint32_t* __restrict__ hist, unsigned ntiles)
{
	__shared__ uint32_t h[RADIX_DIGITS];
	h[threadIdx.x] = 0;
	__syncthreads();
	const unsigned lane = threadIdx.x & 31;
	size_t base = (size_t)blockIdx.x * RADIX_TILE;
	for (int r = 0; r < RADIX_ROUNDS; ++r) {
		size_t i = base + (size_t)r * RADIX_BLOCK + threadIdx.x;
		unsigned d = i < n ? (unsigned)((keys[i] >> shift) & 255u) : 256u;
		unsigned peers = __match_any_sync(0xffffffffu, d);
		if (d < 256u && (__ffs(peers) - 1) == (int)lane) atomicAdd(&h[d], (uint32_t)__popc(peers));
	}
	__syncthreads();
	hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: rank of a key inside its tile = keys with the same digit in
// earlier rounds (running base) + in earlier warps of this round (stamped
// per-warp counts) + in earlier lanes of this warp (match_any mask).
__global__ void __launch_bounds__(RADIX_BLOCK) radix_scatter_kernel(const uint64_t* __restrict__ kin,
                                                                    const uint32_t* __restrict__ vin,
                                                                    uint64_t* __restrict__ kout,
                                                                    uint32_t* __restrict__ vout, size_t n, int shift,
                                                                    const uint32_t* __restrict__ offsets, unsigned ntiles)
{
	constexpr int NW = RADIX_BLOCK / 32;
	__shared__ uint32_t base[RADIX_DIGITS];
	__shared__ uint32_t wcnt[NW][RADIX_DIGITS];
	const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	base[threadIdx.x] = offsets[(size_t)threadIdx.x * ntiles + blockIdx.x];
	for (int i = threadIdx.x; i < NW * RADIX_DIGITS; i += RADIX_BLOCK) (&wcnt[0][0])[i] = 0xffffffffu;
	__syncthreads();
	const unsigned lt = (1u << lane) - 1u;
	size_t tile0 = (size_t)blockIdx.x * RADIX_TILE;
	for (int r = 0; r < RADIX_ROUNDS; ++r) {
		size_t i = tile0 + (size_t)r * RADIX_BLOCK + threadIdx.x;
		bool valid = i < n;
		uint64_t k = valid ? kin[i] : 0ull;
		uint32_t v = valid ? vin[i] : 0u;
		unsigned d = valid ? (unsigned)((k >> shift) & 255u) : 256u;
		unsigned peers = __match_any_sync(0xffffffffu, d);
		unsigned rank = __popc(peers & lt), cnt = __popc(peers);
		bool leader = (__ffs(peers) - 1) == (int)lane;
		if (valid && leader) wcnt[warp][d] = ((unsigned)r << 16) | cnt;
		__syncthreads();
		if (valid) {
			uint32_t off = base[d];
			for (unsigned w = 0; w < warp; ++w) {
				uint32_t c = wcnt[w][d];
				if ((c >> 16) == (unsigned)r) off += c & 0xffffu;
			}
			kout[off + rank] = k;
			vout[off + rank] = v;
		}
		__syncthreads();
		if (valid && leader) atomicAdd(&base[d], cnt);
		__syncthreads();
	}
}

} // namespace

size_t scan_scratch_words(size_t n)
{
	size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
	return nb + 64;
}

void scan_exclusive_u32(const uint32_t* in, uint32_t* out, size_t n, uint32_t* total, uint32_t* scratch,
                        cudaStream_t s)
{
	if (n == 0) {
		if (total) cudaMemsetAsync(total, 0, sizeof(uint32_t), s);
		return;
	}
	size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
	scan_reduce_kernel<<<(unsigned)nb, SCAN_BLOCK, 0, s>>>(in, n, scratch);
	scan_sums_kernel<<<1, SCAN_BLOCK, 0, s>>>(scratch, nb, total);
	scan_apply_kernel<<<(unsigned)nb, SCAN_BLOCK, 0, s>>>(in, out, n, scratch);
}

size_t radix_scratch_words(size_t n)
{
	size_t ntiles = (n + RADIX_TILE - 1) / RADIX_TILE;
	size_t h = ntiles * RADIX_DIGITS;
	return h + scan_scratch_words(h) + 64;
}

int radix_sort_pairs(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt, size_t n,
                     int begin_bit, int end_bit, uint32_t* scratch, cudaStream_t s)
{
	if (n <= 1 || end_bit <= begin_bit) return 0;
	unsigned ntiles = (unsigned)((n + RADIX_TILE - 1) / RADIX_TILE);
	size_t h = (size_t)ntiles * RADIX_DIGITS;
	uint32_t* hist = scratch;
	uint32_t* sc = scratch + h;
	uint64_t *ka = keys, *kb = keys_alt;
	uint32_t *va = vals, *vb = vals_alt;
	int which = 0;
	for (int shift = begin_bit; shift < end_bit; shift += 8) {
		radix_hist_kernel<<<ntiles, RADIX_BLOCK, 0, s>>>(ka, n, shift, hist, ntiles);
		scan_exclusive_u32(hist, hist, h, nullptr, sc, s);
		radix_scatter_kernel<<<ntiles, RADIX_BLOCK, 0, s>>>(ka, va, kb, vb, n, shift, hist, ntiles);
		uint64_t* tk = ka; ka = kb; kb = tk;
		uint32_t* tv = va; va = vb; vb = tv;
		which ^= 1;
	}
	return which;
}

} // namespace lfmm
