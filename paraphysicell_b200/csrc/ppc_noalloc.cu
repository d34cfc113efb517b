// ppc_noalloc.cu — mesh binning that allocates no memory.
//
// Some callers cannot call cudaMalloc at the point where they need the
// mechanics mesh: code that runs under an allocator that forbids hidden
// allocations (a framework's caching allocator or a memory-capped pool),
// real-time loops that must not block on the driver's allocator, or code
// that is not allowed to create a ppc_state at all. ppc_bin_agents_noalloc
// bins agents given in the caller's own device buffers and keeps every
// intermediate (voxel keys, provisional ranks, the per-voxel prefix, per-tile
// totals) in g_noalloc_scratch below, a fixed-size array in device memory.
// Every GPU that loads this library reserves that array until the process
// exits. All calls share it and it keeps the previous call's contents; every
// entry is rewritten before it is read, so nothing has to be cleared between
// calls, but calls whose work overlaps on the GPU (different streams, or
// different host threads on one device) race on it.
//
// The result is the one ppc_update_mechanics_mesh + ppc_get_mesh_bins give:
// per-voxel counts and the agents grouped by voxel in voxel order, in
// descending index inside a voxel (the order of a serial run of the
// reference's counting sort).
#include <cuda_runtime.h>

#include <mutex>

#include "ppc_internal.cuh"

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaTileShift = 12; // 4096 voxels per scan tile
constexpr int kNaTileItems = 16; // voxels per thread in the scan
constexpr int64_t kNaTiles = (PPC_NOALLOC_MAX_VOXELS + 4095) / 4096;

// layout of the scratch, in int32 units
constexpr int64_t kOffKey = 0;
constexpr int64_t kOffRank = kOffKey + PPC_NOALLOC_MAX_AGENTS;
constexpr int64_t kOffTmp = kOffRank + PPC_NOALLOC_MAX_AGENTS;
constexpr int64_t kOffStart = kOffTmp + PPC_NOALLOC_MAX_AGENTS;
constexpr int64_t kOffTile = kOffStart + kNaTiles * 4096 + 64;
constexpr int64_t kScratchInts = kOffTile + kNaTiles + 64;

static __device__ __align__(256) int32_t g_noalloc_scratch[kScratchInts];

struct na_mesh
{
	double mins[3], maxs[3], shape[3];
	int32_t grid[3];
	int32_t dims;
	int32_t nvox;
};

__device__ __forceinline__ int na_axis(double x, const na_mesh& m, int d)
{
	const double q = (x - m.mins[d]) / m.shape[d];
	if (!(q == q) || q <= 0.0)
		return 0;
	if (q >= (double)m.grid[d])
		return m.grid[d] - 1;
	return (int)q;
}

__global__ void k_na_count(const double* __restrict__ pos, int n, na_mesh m, int32_t* counts, int32_t* scratch)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const double x = pos[(int64_t)i * m.dims];
	const double y = m.dims >= 2 ? pos[(int64_t)i * m.dims + 1] : 0.0;
	const double z = m.dims >= 3 ? pos[(int64_t)i * m.dims + 2] : 0.0;
	const int c0 = na_axis(x, m, 0);
	const int c1 = m.dims >= 2 ? na_axis(y, m, 1) : 0;
	const int c2 = m.dims >= 3 ? na_axis(z, m, 2) : 0;
	const int32_t key = c0 + m.grid[0] * (c1 + m.grid[1] * c2);
	const int32_t rank = atomicAdd(counts + key, 1);
	scratch[kOffKey + i] = key;
	scratch[kOffRank + i] = rank;
}

__device__ __forceinline__ int na_block_scan(int x, int& total)
{
	__shared__ int sums[32];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	int incl = x;
	for (int o = 1; o < 32; o <<= 1)
	{
		const int y = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= o)
			incl += y;
	}
	if (lane == 31)
		sums[warp] = incl;
	__syncthreads();
	const int nw = blockDim.x >> 5;
	if (warp == 0)
	{
		int w = lane < nw ? sums[lane] : 0;
		for (int o = 1; o < 32; o <<= 1)
		{
			const int y = __shfl_up_sync(0xffffffffu, w, o);
			if (lane >= o)
				w += y;
		}
		if (lane < nw)
			sums[lane] = w;
	}
	__syncthreads();
	total = sums[nw - 1];
	const int excl = incl - x + (warp > 0 ? sums[warp - 1] : 0);
	__syncthreads();
	return excl;
}

__global__ void k_na_reduce(const int32_t* counts, int nvox, int32_t* scratch)
{
	const int64_t i0 = ((int64_t)blockIdx.x << kNaTileShift) + (int64_t)threadIdx.x * kNaTileItems;
	int sum = 0;
	for (int k = 0; k < kNaTileItems; k++)
		if (i0 + k < nvox)
			sum += counts[i0 + k];
	int total;
	na_block_scan(sum, total);
	if (threadIdx.x == 0)
		scratch[kOffTile + blockIdx.x] = total;
}

__global__ void k_na_scan(const int32_t* counts, int nvox, int32_t* scratch)
{
	const int b = blockIdx.x;
	int part = 0;
	for (int k = threadIdx.x; k < b; k += blockDim.x)
		part += scratch[kOffTile + k];
	int base;
	na_block_scan(part, base);
	const int64_t i0 = ((int64_t)b << kNaTileShift) + (int64_t)threadIdx.x * kNaTileItems;
	int c[kNaTileItems];
	int sum = 0;
	for (int k = 0; k < kNaTileItems; k++)
	{
		c[k] = i0 + k < nvox ? counts[i0 + k] : 0;
		sum += c[k];
	}
	int total;
	int run = base + na_block_scan(sum, total);
	for (int k = 0; k < kNaTileItems; k++)
		if (i0 + k < nvox)
		{
			scratch[kOffStart + i0 + k] = run;
			run += c[k];
		}
	if (b == gridDim.x - 1 && threadIdx.x == blockDim.x - 1)
		scratch[kOffStart + nvox] = run;
}

__global__ void k_na_scatter(int n, int32_t* scratch)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const int32_t key = scratch[kOffKey + i];
	const int32_t rank = scratch[kOffRank + i];
	const int32_t st = scratch[kOffStart + key];
	scratch[kOffTmp + st + rank] = i;
}

// final place inside the voxel: descending agent index. Each agent counts
// the larger indices of its voxel, so a voxel of c agents costs c^2 loads:
// nothing at tissue densities (a few agents per voxel), about 1.7e10 loads
// for the degenerate case of all PPC_NOALLOC_MAX_AGENTS agents in one voxel.
__global__ void k_na_order(int n, const int32_t* scratch, int32_t* agents)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n)
		return;
	const int32_t key = scratch[kOffKey + i];
	const int32_t st = scratch[kOffStart + key];
	const int32_t c = scratch[kOffStart + key + 1] - st;
	int rank = 0;
	for (int u = 0; u < c; u++)
		rank += scratch[kOffTmp + st + u] > i;
	agents[st + rank] = i;
}

std::mutex g_na_mutex;
void* g_na_ptr[256] = {};

} // namespace

extern "C" int ppc_bin_agents_noalloc(const ppc_mesh* mesh, const double* positions, int32_t count,
									  int32_t* voxel_counts, int32_t* agents, void* cuda_stream)
{
	if (!mesh || count < 0 || (count > 0 && (!positions || !agents)) || !voxel_counts || mesh->dims < 1
		|| mesh->dims > 3)
	{
		ppc::set_error("ppc_bin_agents_noalloc: null buffer or dims outside 1..3");
		return PPC_ERR_ARG;
	}
	na_mesh m {};
	m.dims = mesh->dims;
	// grid sizes in 64-bit arithmetic, each axis and the running product
	// checked against the scratch's voxel limit before the next multiply, so
	// no extent of the 32-bit mesh fields can wrap the voxel count
	int64_t nvox = 1;
	bool too_many = false;
	for (int d = 0; d < 3; d++)
	{
		m.mins[d] = mesh->bounding_box_mins[d];
		m.maxs[d] = mesh->bounding_box_maxs[d];
		m.shape[d] = mesh->voxel_shape[d];
		int64_t g = 1;
		if (d < mesh->dims)
		{
			if (mesh->voxel_shape[d] <= 0 || mesh->bounding_box_maxs[d] < mesh->bounding_box_mins[d])
			{
				ppc::set_error("ppc_bin_agents_noalloc: invalid mesh");
				return PPC_ERR_ARG;
			}
			const int64_t extent = (int64_t)mesh->bounding_box_maxs[d] - (int64_t)mesh->bounding_box_mins[d];
			g = (extent + mesh->voxel_shape[d] - 1) / mesh->voxel_shape[d];
		}
		g = g < 1 ? 1 : g;
		too_many = too_many || g > PPC_NOALLOC_MAX_VOXELS;
		nvox = too_many ? PPC_NOALLOC_MAX_VOXELS + 1 : nvox * g;
		too_many = too_many || nvox > PPC_NOALLOC_MAX_VOXELS;
		m.grid[d] = (int32_t)(too_many ? 1 : g);
	}
	if (count > PPC_NOALLOC_MAX_AGENTS || too_many)
	{
		ppc::set_error("ppc_bin_agents_noalloc: at most " + std::to_string(PPC_NOALLOC_MAX_AGENTS) + " agents and "
					   + std::to_string(PPC_NOALLOC_MAX_VOXELS) + " voxels fit its fixed scratch (asked for "
					   + std::to_string(count) + " agents, "
					   + (too_many ? std::string("more than the limit of") : std::to_string(nvox)) + " voxels)");
		return PPC_ERR_CAPACITY;
	}
	m.nvox = (int32_t)nvox;

	// the scratch's device address, looked up once per device with that
	// device current (the symbol's host-side name is only a stand-in)
	int dev = 0;
	cudaError_t e = cudaGetDevice(&dev);
	if (e != cudaSuccess || dev < 0 || dev >= 256)
		return e != cudaSuccess ? ppc::cuda_fail(e, "cudaGetDevice") : PPC_ERR_NO_DEVICE;
	int32_t* scratch = nullptr;
	{
		std::lock_guard<std::mutex> lock(g_na_mutex);
		if (!g_na_ptr[dev])
		{
			void* p = nullptr;
			e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
			if (e != cudaSuccess)
				return ppc::cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
			g_na_ptr[dev] = p;
		}
		scratch = static_cast<int32_t*>(g_na_ptr[dev]);
	}

	cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
	PPC_CUDA(cudaMemsetAsync(voxel_counts, 0, sizeof(int32_t) * nvox, st));
	if (count == 0)
		return PPC_OK;
	const int b = (count + kNaThreads - 1) / kNaThreads;
	const int tiles = (int)((nvox + 4095) / 4096);
	k_na_count<<<b, kNaThreads, 0, st>>>(positions, count, m, voxel_counts, scratch);
	k_na_reduce<<<tiles, kNaThreads, 0, st>>>(voxel_counts, m.nvox, scratch);
	k_na_scan<<<tiles, kNaThreads, 0, st>>>(voxel_counts, m.nvox, scratch);
	k_na_scatter<<<b, kNaThreads, 0, st>>>(count, scratch);
	k_na_order<<<b, kNaThreads, 0, st>>>(count, scratch, agents);
	PPC_CUDA(cudaGetLastError());
	return PPC_OK;
}
