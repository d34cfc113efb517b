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
 * Random walks: the reference's own construction (src/solver/host/
 * solver_helper.h:82-86,160-165,250-267): in 1-D a sign from one uniform
 * draw; in 2-D an angle theta = 2 pi u and the direction (cos theta,
 * sin theta); in 3-D theta as in 2-D, z = 2 u' - 1 and the direction
 * (cos theta sqrt(1 - z^2), sin theta sqrt(1 - z^2), z). The draws are mapped
 * to their ranges with the operations of std::uniform_real_distribution
 * (u (b - a) + a). cos and sin are this file's own ppc_sincos (Cody-Waite
 * reduction and Taylor polynomials, below), so host and device produce the
 * same bits; libm and CUDA differ from each other, and from it, in the last
 * bit now and then.
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
#define PPC_DRAW_WALK 16u		 /* division offset: theta, then z (3-D) */
#define PPC_DRAW_ORIENTATION 96u /* daughter orientation: theta, then z (3-D) */
#define PPC_DRAW_INTERACTION 1048576u /* + neighbour position, cell-cell interactions */
#define PPC_DRAW_MOTILITY 2097152u	/* persistence draw; the walk's theta and z follow */

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

/* Sine and cosine of theta for |theta| <= 2^19 (the random walks pass
 * theta in [0, 2 pi)).
 *
 * Reduction: k = floor(theta 2/pi + 1/2), r = theta - k pi/2 with pi/2 split
 * into three parts (W. J. Cody and W. Waite, "Software Manual for the
 * Elementary Functions", 1980): P1 and P2 are pi/2 and the remainder rounded
 * to 33 significant bits, so k P1 and k P2 are exact for |k| < 2^20, and P3 is
 * the next remainder rounded to 53 bits; all three were derived from the
 * decimal expansion of pi in exact rational arithmetic. |r| <= pi/4 plus an
 * ulp.
 * Polynomials: the Taylor series of sin and cos about 0 through the terms in
 * r^19 and r^18, whose truncation error on |r| <= pi/4 is below 1e-19;
 * coefficients 1/n! (n! is exact in double for n <= 22, the quotients are
 * correctly rounded), evaluated by Horner's rule.
 * Result: sin/cos(r) mapped to theta's quadrant k mod 4. Accurate to about
 * one ulp; every operation is a correctly rounded IEEE operation, so the host
 * and the device agree bit for bit. */
PPC_HD void ppc_sincos(double theta, double* sn, double* cs)
{
	const double two_over_pi = 0x1.45f306dc9c883p-1;
	const double P1 = 0x1.921fb544p+0;
	const double P2 = 0x1.0b4611a6p-34;
	const double P3 = 0x1.3198a2e037073p-69;
	const double kd = floor(PPC_ADD(PPC_MUL(theta, two_over_pi), 0.5));
	const double r = PPC_SUB(PPC_SUB(PPC_SUB(theta, PPC_MUL(kd, P1)), PPC_MUL(kd, P2)), PPC_MUL(kd, P3));
	const double r2 = PPC_MUL(r, r);
	/* sin r = r + r r2 (-1/3! + r2 (1/5! - ...)) */
	double ps = -1.0 / 121645100408832000.0; /* -1/19! */
	ps = PPC_ADD(PPC_MUL(ps, r2), 1.0 / 355687428096000.0);
	ps = PPC_ADD(PPC_MUL(ps, r2), -1.0 / 1307674368000.0);
	ps = PPC_ADD(PPC_MUL(ps, r2), 1.0 / 6227020800.0);
	ps = PPC_ADD(PPC_MUL(ps, r2), -1.0 / 39916800.0);
	ps = PPC_ADD(PPC_MUL(ps, r2), 1.0 / 362880.0);
	ps = PPC_ADD(PPC_MUL(ps, r2), -1.0 / 5040.0);
	ps = PPC_ADD(PPC_MUL(ps, r2), 1.0 / 120.0);
	ps = PPC_ADD(PPC_MUL(ps, r2), -1.0 / 6.0);
	const double s = PPC_ADD(r, PPC_MUL(PPC_MUL(r, r2), ps));
	/* cos r = 1 + r2 (-1/2! + r2 (1/4! - ...)) */
	double pc = -1.0 / 6402373705728000.0; /* -1/18! */
	pc = PPC_ADD(PPC_MUL(pc, r2), 1.0 / 20922789888000.0);
	pc = PPC_ADD(PPC_MUL(pc, r2), -1.0 / 87178291200.0);
	pc = PPC_ADD(PPC_MUL(pc, r2), 1.0 / 479001600.0);
	pc = PPC_ADD(PPC_MUL(pc, r2), -1.0 / 3628800.0);
	pc = PPC_ADD(PPC_MUL(pc, r2), 1.0 / 40320.0);
	pc = PPC_ADD(PPC_MUL(pc, r2), -1.0 / 720.0);
	pc = PPC_ADD(PPC_MUL(pc, r2), 1.0 / 24.0);
	pc = PPC_ADD(PPC_MUL(pc, r2), -0.5);
	const double c = PPC_ADD(1.0, PPC_MUL(r2, pc));
	switch ((int)((long long)kd & 3))
	{
	case 0:
		*sn = s;
		*cs = c;
		break;
	case 1:
		*sn = c;
		*cs = -s;
		break;
	case 2:
		*sn = -s;
		*cs = -c;
		break;
	default:
		*sn = -c;
		*cs = s;
		break;
	}
}

/* position_helper<dims>::random_walk (reference: src/solver/host/
 * solver_helper.h:82-86,160-165,250-267) with draws k0 (the sign, or theta)
 * and k0 + 1 (z, 3-D only) of (seed, epoch, replicate, slot); writes
 * w[0..dims-1]. The 3-D walk restricted to the plane is the 2-D walk with
 * w[2] = 0, as in the reference. */
PPC_HD void ppc_random_walk(int dims, uint64_t seed, uint64_t epoch, uint64_t replicate, uint64_t slot, uint64_t k0,
							double* w)
{
	const double two_pi = 6.283185307179586; /* 2 std::numbers::pi_v<double>, exact */
	const double u = ppc_uniform(seed, epoch, replicate, slot, k0);
	if (dims == 1)
	{
		w[0] = u < 0.5 ? -1.0 : 1.0;
		return;
	}
	/* uniform(0, 2 pi) = u (2 pi - 0) + 0 */
	const double theta = PPC_ADD(PPC_MUL(u, PPC_SUB(two_pi, 0.0)), 0.0);
	double sn, cs;
	ppc_sincos(theta, &sn, &cs);
	if (dims == 2)
	{
		w[0] = cs;
		w[1] = sn;
		return;
	}
	/* uniform(-1, 1) = u' (1 - (-1)) + (-1) */
	const double z = PPC_ADD(PPC_MUL(ppc_uniform(seed, epoch, replicate, slot, k0 + 1u), 2.0), -1.0);
	const double rr = PPC_SQRT(PPC_SUB(1.0, PPC_MUL(z, z)));
	w[0] = PPC_MUL(cs, rr);
	w[1] = PPC_MUL(sn, rr);
	w[2] = z;
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
