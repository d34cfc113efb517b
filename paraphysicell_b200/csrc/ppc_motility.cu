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

// normalize (reference: src/solver/host/solver_helper.h:30-45)
template <int DIMS>
__device__ __forceinline__ void normalize(double* x)
{
	double length = 0;
	for (int d = 0; d < DIMS; d++)
		length += x[d] * x[d];
	length = sqrt(length);
	for (int d = 0; d < DIMS; d++)
		x[d] = length > kZeroThreshold ? x[d] / length : 0;
}

// agent::nearest_gradient of substrate q at position p: the gradient of the
// diffusion voxel holding p (truncation of (x - min) / voxel edge, clamped
// into the grid, as for the mechanics mesh)
template <int DIMS>
__device__ __forceinline__ void nearest_gradient(const mot_fields& m, const double4& p, int q, double* g)
{
	int c[3] = { 0, 0, 0 };
	for (int d = 0; d < DIMS; d++)
	{
		const double x = d == 0 ? p.x : (d == 1 ? p.y : p.z);
		const double f = (x - m.gmins[d]) / m.gshape[d];
		int k = f > 0 ? (int)f : 0;
		c[d] = k < m.ggrid[d] ? k : m.ggrid[d] - 1;
	}
	const int64_t vox = c[0] + (int64_t)m.ggrid[0] * (c[1] + (int64_t)m.ggrid[1] * c[2]);
	const double* row = m.grad + (vox * m.gS + q) * 3;
	for (int d = 0; d < DIMS; d++)
		g[d] = row[d];
}

// the standard direction-update rules (reference:
// src/original/core/standard_models.cpp:542-583)
template <int DIMS>
__device__ void direction_rule(const view& v, const mot_fields& m, int i, int rule)
{
	const double4 p = v.pos[m.cur][m.base + i]; // the position the step started from
	double dir[DIMS];
	if (rule == PPC_DIRECTION_CHEMOTAXIS)
	{
		double g[DIMS];
		nearest_gradient<DIMS>(m, p, m.chemo_index[i], g);
		for (int d = 0; d < DIMS; d++)
			dir[d] = g[d] * m.chemo_dir[i];
	}
	else
	{
		for (int d = 0; d < DIMS; d++)
			dir[d] = 0;
		for (int q = 0; q < m.gS; q++)
		{
			double g[DIMS];
			nearest_gradient<DIMS>(m, p, q, g);
			if (rule == PPC_DIRECTION_ADVANCED_CHEMOTAXIS_NORMALIZED)
				normalize<DIMS>(g);
			const double w = q < m.S ? m.sens[(int64_t)i * m.S + q] : 0.0;
			for (int d = 0; d < DIMS; d++)
				dir[d] += g[d] * w;
		}
	}
	normalize<DIMS>(dir);
	for (int d = 0; d < DIMS; d++)
		m.direction[(int64_t)i * DIMS + d] = dir[d];
}

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
		// the direction-update callback runs after the walk is drawn
		// (position_solver.cpp:133-136)
		const int rule = m.rule ? (int)m.rule[i] : (int)PPC_DIRECTION_NONE;
		if (rule != PPC_DIRECTION_NONE && m.grad)
			direction_rule<DIMS>(v, m, i, rule);
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
