// Motility on the device (reference: src/solver/host/position_solver.cpp:115-145,198-212,288-314,
// src/solver/host/solver_helper.h:82-101,160-182,250-287). One thread per agent: a motile agent
// redraws its direction with probability dt / persistence_time, mixes it with its migration
// bias direction, scales the result to its migration speed and adds it to its velocity. The
// direction is the reference's random walk (an angle, and z in 3-D) from counter-based draws,
// with the sine and cosine of ppc_draws.h, bit-identical on host and device.

#include <cuda_runtime.h>

#include "../../include/ppc_draws.h"
#include "ppc_internal.cuh"

namespace ppc {
namespace {

constexpr int kMotThreads = 256;
constexpr double kZeroThreshold = 1e-16; // reference: solver_helper.h:12

__device__ __forceinline__ double& comp_ref(double4& v, int d) { return d == 0 ? v.x : (d == 1 ? v.y : v.z); }

template <int DIMS>
__global__ void __launch_bounds__(kMotThreads) k_motility(view v, mot_fields m)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= m.n || m.motile[i] == 0)
		return;
	double mv[DIMS];
	for (int d = 0; d < DIMS; d++)
		mv[d] = m.vector[(int64_t)i * DIMS + d];
	if (ppc_uniform(v.seed, m.epoch, (uint64_t)m.replicate, (uint64_t)i, PPC_DRAW_MOTILITY) < m.dt / m.persistence[i])
	{
		double walk[3] = { 0, 0, 0 };
		// the reference's walk is planar for every 3-D agent (its bool
		// parameter receives the restrict_to_2d array pointer,
		// position_solver.cpp:131); per_agent reads each agent's flag instead
		const bool planar = DIMS == 3 && (m.per_agent ? m.restrict2d[i] != 0 : true);
		ppc_random_walk(planar ? 2 : DIMS, v.seed, m.epoch, (uint64_t)m.replicate, (uint64_t)i, PPC_DRAW_MOTILITY + 1u,
						walk);
		const double bias = m.bias[i];
		for (int d = 0; d < DIMS; d++)
			mv[d] = (1 - bias) * walk[d] + bias * m.direction[(int64_t)i * DIMS + d];
		// normalize_and_scale
		double len2 = mv[0] * mv[0];
		for (int d = 1; d < DIMS; d++)
			len2 = len2 + mv[d] * mv[d];
		const double length = DIMS == 1 ? fabs(mv[0]) : sqrt(len2);
		const double scale = m.speed[i];
		for (int d = 0; d < DIMS; d++)
			mv[d] = length > kZeroThreshold ? mv[d] * scale / length : 0;
		for (int d = 0; d < DIMS; d++)
			m.vector[(int64_t)i * DIMS + d] = mv[d];
	}
	const int s = m.base + i;
	double4 vel = v.vel[s];
	for (int d = 0; d < DIMS; d++)
		comp_ref(vel, d) += mv[d];
	v.vel[s] = vel;
}

} // namespace

int launch_motility(ppc_state* s, const mot_fields& m)
{
	if (m.n == 0)
		return PPC_OK;
	const int b = blocks_for(m.n, kMotThreads);
	if (s->dims == 1)
		k_motility<1><<<b, kMotThreads, 0, PPC_LAUNCH(s)>>>(s->v, m);
	else if (s->dims == 2)
		k_motility<2><<<b, kMotThreads, 0, PPC_LAUNCH(s)>>>(s->v, m);
	else
		k_motility<3><<<b, kMotThreads, 0, PPC_LAUNCH(s)>>>(s->v, m);
	PPC_CUDA(cudaGetLastError());
	return PPC_OK;
}

} // namespace ppc
