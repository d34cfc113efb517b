/*
 * ppc_draws.h — deterministic random draws and the cube root used by division.
 *
 * The reference draws its random numbers from a thread_local std::mt19937
 * (reference: src/random.cpp:8-26), so a multi-threaded run is not
 * reproducible and a GPU cannot replay it. This build replaces every draw of
 * the mechanics/division path by a counter-based stream: draw k of agent slot
 * i in replicate r at event epoch e is a pure function of (seed, e, r, i, k).
 * Host code (the CPU oracle) and device code evaluate the same integer hash
 * and the same sequence of correctly rounded IEEE operations, so both produce
 * bit-identical values.
 *
 * Hash: the SplitMix64 output function (G. Steele, D. Lea, C. Flood,
 * "Fast splittable pseudorandom number generators", OOPSLA 2014), applied in
 * a chain over the counter words.
 *
 * Unit vectors: Marsaglia's rejection method for points on the sphere
 * (G. Marsaglia, "Choosing a point from the surface of a sphere", Ann. Math.
 * Statist. 43, 1972) in 3-D and the same rejection square for the circle in
 * 2-D; they replace the reference's angle-based random walk
 * (src/solver/host/solver_helper.h:82-86,160-165,250-267), which needs cos/sin
 * whose last bit differs between libm and CUDA. Both give directions uniform
 * on the sphere/circle.
 *
 * Cube root: Newton's iteration for y^3 = t on a range-reduced argument, with
 * a last step whose residual uses exact FMA products. The reference uses
 * std::cbrt (src/solver/host/interactions_solver.cpp:89-96); this
 * deterministic version agrees with glibc's to within one ulp and is
 * identical on host and device (FMA is correctly rounded on both).
 *
 * Host compilation must not contract a*b+c into FMA (-ffp-contract=off); on
 * the device the operations are spelled with the _rn intrinsics.
 */
#ifndef PPC_DRAWS_H
#define PPC_DRAWS_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
	#define PPC_HD __host__ __device__ __forceinline__
#else
	#define PPC_HD static inline
#endif

#if defined(__CUDA_ARCH__)
	#define PPC_MUL(a, b) __dmul_rn((a), (b))
	#define PPC_ADD(a, b) __dadd_rn((a), (b))
	#define PPC_SUB(a, b) __dsub_rn((a), (b))
	#define PPC_DIV(a, b) __ddiv_rn((a), (b))
	#define PPC_SQRT(a) __dsqrt_rn((a))
	#define PPC_FMA(a, b, c) __fma_rn((a), (b), (c))
#else
	#include <math.h>
	#define PPC_MUL(a, b) ((a) * (b))
	#define PPC_ADD(a, b) ((a) + (b))
	#define PPC_SUB(a, b) ((a) - (b))
	#define PPC_DIV(a, b) ((a) / (b))
	#define PPC_SQRT(a) sqrt((a))
	#define PPC_FMA(a, b, c) fma((a), (b), (c))
#endif

/* draw slots k used by the mechanics path */
#define PPC_DRAW_DEATH 0u
#define PPC_DRAW_DIVIDE 1u
#define PPC_DRAW_WALK 16u		 /* 2 per attempt, up to PPC_DRAW_ATTEMPTS attempts */
#define PPC_DRAW_ORIENTATION 96u /* 2 per attempt */
#define PPC_DRAW_ATTEMPTS 32u
#define PPC_DRAW_INTERACTION 1048576u /* + neighbour position, cell-cell interactions */
#define PPC_DRAW_MOTILITY 2097152u	/* persistence draw; the direction's draws follow */

PPC_HD uint64_t ppc_mix64(uint64_t z)
{
	z += 0x9E3779B97F4A7C15ull;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

PPC_HD uint64_t ppc_hash(uint64_t seed, uint64_t epoch, uint64_t replicate, uint64_t slot, uint64_t k)
{
	uint64_t h = ppc_mix64(seed);
	h = ppc_mix64(h ^ epoch);
	h = ppc_mix64(h ^ replicate);
	h = ppc_mix64(h ^ slot);
	h = ppc_mix64(h ^ k);
	return h;
}

/* uniform double in [0, 1) with 53 random bits */
PPC_HD double ppc_uniform(uint64_t seed, uint64_t epoch, uint64_t replicate, uint64_t slot, uint64_t k)
{
	return (double)(ppc_hash(seed, epoch, replicate, slot, k) >> 11) * (1.0 / 9007199254740992.0);
}

/* Uniform random direction in `dims` dimensions written to w[0..dims-1],
 * from draws k0, k0+1, ... of (seed, epoch, replicate, slot). */
PPC_HD void ppc_unit_vector(int dims, uint64_t seed, uint64_t epoch, uint64_t replicate, uint64_t slot, uint64_t k0,
							double* w)
{
	if (dims == 1)
	{
		/* reference: solver_helper.h:82-86, walk = rand < 0.5 ? -1 : 1 */
		double u = ppc_uniform(seed, epoch, replicate, slot, k0);
		w[0] = u < 0.5 ? -1.0 : 1.0;
		return;
	}
	for (uint32_t t = 0; t < PPC_DRAW_ATTEMPTS; t++)
	{
		double a = PPC_SUB(PPC_MUL(2.0, ppc_uniform(seed, epoch, replicate, slot, k0 + 2 * t)), 1.0);
		double b = PPC_SUB(PPC_MUL(2.0, ppc_uniform(seed, epoch, replicate, slot, k0 + 2 * t + 1)), 1.0);
		double s = PPC_ADD(PPC_MUL(a, a), PPC_MUL(b, b));
		if (s >= 1.0 || s == 0.0)
			continue;
		if (dims == 2)
		{
			double l = PPC_SQRT(s);
			w[0] = PPC_DIV(a, l);
			w[1] = PPC_DIV(b, l);
		}
		else
		{
			double f = PPC_MUL(2.0, PPC_SQRT(PPC_SUB(1.0, s)));
			w[0] = PPC_MUL(a, f);
			w[1] = PPC_MUL(b, f);
			w[2] = PPC_SUB(1.0, PPC_MUL(2.0, s));
		}
		return;
	}
	/* probability of reaching here is (1 - pi/4)^32 < 1e-21 */
	w[0] = 0.0;
	w[1] = 0.0;
	if (dims == 3)
		w[2] = 1.0;
	else
		w[0] = 1.0;
}

PPC_HD uint64_t ppc_d2u(double x)
{
	uint64_t u;
	memcpy(&u, &x, sizeof u);
	return u;
}

PPC_HD double ppc_u2d(uint64_t u)
{
	double x;
	memcpy(&x, &u, sizeof x);
	return x;
}

/* Cube root of a positive normal double by Newton's method on the mantissa
 * range [1, 8), scaled back by an exact power of two. Zero, negative,
 * subnormal and non-finite inputs are handled by sign symmetry or returned
 * unchanged. */
PPC_HD double ppc_cbrt(double x)
{
	if (!(x == x) || x == 0.0)
		return x;
	int neg = x < 0.0;
	double a = neg ? -x : x;
	uint64_t bits = ppc_d2u(a);
	int64_t e = (int64_t)((bits >> 52) & 0x7ff);
	if (e == 0 || e == 0x7ff)
		return x; /* subnormal or infinite: outside the range division produces */
	e -= 1023;
	int64_t q = e >= 0 ? e / 3 : -((-e + 2) / 3);
	int64_t r = e - 3 * q; /* 0, 1 or 2 */
	double m = ppc_u2d((bits & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
	double t = r == 0 ? m : (r == 1 ? PPC_MUL(m, 2.0) : PPC_MUL(m, 4.0)); /* exact, t in [1, 8) */
	/* chord of cbrt on [1, 8) lies below the curve; Newton from there
	   overshoots once and then decreases monotonically to the root */
	double y = PPC_ADD(1.0, PPC_DIV(PPC_SUB(t, 1.0), 7.0));
	for (int it = 0; it < 6; it++)
	{
		double y2 = PPC_MUL(y, y);
		y = PPC_SUB(y, PPC_DIV(PPC_SUB(y, PPC_DIV(t, y2)), 3.0));
	}
	/* one more Newton step with the residual t - y^3 formed from exact
	   products (FMA error terms), which removes the rounding error of the
	   plain iteration */
	{
		double p = PPC_MUL(y, y);
		double ep = PPC_FMA(y, y, -p); /* y*y = p + ep exactly */
		double c = PPC_MUL(p, y);
		double ec = PPC_FMA(p, y, -c); /* p*y = c + ec exactly */
		double res = PPC_SUB(PPC_SUB(PPC_SUB(t, c), ec), PPC_MUL(ep, y));
		y = PPC_ADD(y, PPC_DIV(res, PPC_MUL(3.0, p)));
	}
	double scale = ppc_u2d((uint64_t)(q + 1023) << 52);
	double res = PPC_MUL(y, scale);
	return neg ? -res : res;
}

#endif /* PPC_DRAWS_H */
