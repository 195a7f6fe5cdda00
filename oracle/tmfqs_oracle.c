/*
 * CPU oracle for the TMFQS dense path -- test infrastructure only.
 *
 * Plain-C restatement of the reference's Dense backend
 * (src/tmfqs/storage/dense/dense_state_backend.cpp), block gate engine
 * (include/tmfqs/storage/gate_block_apply.h), register overlay and cached
 * sum (src/tmfqs/register/quantum_register.cpp), circuit builders
 * (src/tmfqs/circuit/circuit.cpp) and RNG (include/tmfqs/core/random.h,
 * libstdc++ std::mt19937 + std::generate_canonical).
 *
 * Build with -ffp-contract=off: every expression below is evaluated as
 * separately rounded double operations in the reference's source order.
 * Only tests/, the smoke check and bench.py's CPU-baseline leg use this.
 */
#include "tmfqs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI 3.14159265358979323846 /* kPi, include/tmfqs/core/constants.h:6 */

/* Bit mask of qubit q (MSB-first), backend_validation.h:37-39. */
static inline uint64_t qmask(unsigned n, unsigned q) { return (uint64_t)1 << (n - q - 1u); }

/* ---------------------------------------------------------------------- */
/* Dense backend kernels                                                  */
/* ---------------------------------------------------------------------- */

/* Pair iteration (s0, s0 + mask), pair_kernel_executor.h:42-51. */
#define FOR_EACH_PAIR(N, mask, s0, s1, ...)                                   \
	do {                                                                       \
		const uint64_t stride_ = (mask) << 1;                                  \
		for(uint64_t base_ = 0; base_ < (N); base_ += stride_) {               \
			for(uint64_t off_ = 0; off_ < (mask); ++off_) {                    \
				const uint64_t s0 = base_ + off_;                              \
				const uint64_t s1 = s0 + (mask);                               \
				__VA_ARGS__                                                    \
			}                                                                  \
		}                                                                      \
	} while(0)

/* DenseStateBackend::applyHadamard, dense_state_backend.cpp:255-274. */
void or_dense_h(double *a, unsigned n, unsigned q) {
	const uint64_t N = (uint64_t)1 << n;
	const uint64_t m = qmask(n, q);
	const double inv = 1.0 / sqrt(2.0);
	FOR_EACH_PAIR(N, m, s0, s1, {
		double *a0 = a + 2 * s0;
		double *a1 = a + 2 * s1;
		const double ar = a0[0], ai = a0[1], br = a1[0], bi = a1[1];
		if(ar == 0.0 && ai == 0.0 && br == 0.0 && bi == 0.0) continue;
		a0[0] = (ar + br) * inv;
		a0[1] = (ai + bi) * inv;
		a1[0] = (ar - br) * inv;
		a1[1] = (ai - bi) * inv;
	});
}

/* DenseStateBackend::applyPauliX, dense_state_backend.cpp:276-287. */
void or_dense_x(double *a, unsigned n, unsigned q) {
	const uint64_t N = (uint64_t)1 << n;
	const uint64_t m = qmask(n, q);
	FOR_EACH_PAIR(N, m, s0, s1, {
		double *a0 = a + 2 * s0;
		double *a1 = a + 2 * s1;
		if(a0[0] == a1[0] && a0[1] == a1[1]) continue;
		double t = a0[0]; a0[0] = a1[0]; a1[0] = t;
		t = a0[1]; a0[1] = a1[1]; a1[1] = t;
	});
}

/* DenseStateBackend::applyControlledNot, dense_state_backend.cpp:306-319. */
void or_dense_cnot(double *a, unsigned n, unsigned c, unsigned t) {
	const uint64_t N = (uint64_t)1 << n;
	const uint64_t cm = qmask(n, c);
	const uint64_t tm = qmask(n, t);
	FOR_EACH_PAIR(N, tm, s0, s1, {
		if((s0 & cm) == 0) continue;
		double *a0 = a + 2 * s0;
		double *a1 = a + 2 * s1;
		if(a0[0] == a1[0] && a0[1] == a1[1]) continue;
		double x = a0[0]; a0[0] = a1[0]; a1[0] = x;
		x = a0[1]; a0[1] = a1[1]; a1[1] = x;
	});
}

/* DenseStateBackend::applyControlledPhaseShift, dense_state_backend.cpp:289-304. */
void or_dense_cphase(double *a, unsigned n, unsigned c, unsigned t, double theta) {
	const uint64_t N = (uint64_t)1 << n;
	const uint64_t cm = qmask(n, c);
	const uint64_t tm = qmask(n, t);
	const double pr = cos(theta);
	const double pi = sin(theta);
	FOR_EACH_PAIR(N, tm, s0, s1, {
		(void)s0;
		if((s1 & cm) == 0) continue;
		double *a1 = a + 2 * s1;
		const double re = a1[0], im = a1[1];
		if(re == 0.0 && im == 0.0) continue;
		a1[0] = pr * re - pi * im;
		a1[1] = pr * im + pi * re;
	});
}

/* DenseStateBackend::phaseFlipBasisState, dense_state_backend.cpp:205-211. */
void or_dense_phase_flip(double *a, uint64_t s) {
	a[2 * s] = -a[2 * s];
	a[2 * s + 1] = -a[2 * s + 1];
}

/* DenseStateBackend::inversionAboutMean(Amplitude), dense_state_backend.cpp:230-240. */
void or_dense_inversion_mean(double *a, unsigned n, double mre, double mim) {
	const uint64_t N = (uint64_t)1 << n;
	for(uint64_t s = 0; s < N; ++s) {
		const double re = a[2 * s], im = a[2 * s + 1];
		a[2 * s] = 2.0 * mre - re;
		a[2 * s + 1] = 2.0 * mim - im;
	}
}

/* DenseStateBackend::inversionAboutMean(), dense_state_backend.cpp:213-228. */
void or_dense_inversion(double *a, unsigned n) {
	const uint64_t N = (uint64_t)1 << n;
	double sr = 0.0, si = 0.0;
	for(uint64_t s = 0; s < N; ++s) {
		sr += a[2 * s];
		si += a[2 * s + 1];
	}
	or_dense_inversion_mean(a, n, sr / (double)N, si / (double)N);
}

/* DenseStateBackend::applyAffineTransform, dense_state_backend.cpp:242-253. */
void or_dense_affine(double *a, unsigned n, double sre, double sim, double bre, double bim) {
	const uint64_t N = (uint64_t)1 << n;
	for(uint64_t s = 0; s < N; ++s) {
		const double re = a[2 * s], im = a[2 * s + 1];
		a[2 * s] = sre * re - sim * im + bre;
		a[2 * s + 1] = sre * im + sim * re + bim;
	}
}

/* DenseStateBackend::totalProbability, dense_state_backend.cpp:161-171. */
double or_dense_total_probability(const double *a, unsigned n) {
	const uint64_t N = (uint64_t)1 << n;
	double sum = 0.0;
	for(uint64_t s = 0; s < N; ++s) sum += a[2 * s] * a[2 * s] + a[2 * s + 1] * a[2 * s + 1];
	return sum;
}

/* DenseStateBackend::sampleMeasurement, dense_state_backend.cpp:173-188. */
int or_dense_sample(const double *a, unsigned n, double rnd, uint64_t *out) {
	if(rnd < 0.0 || rnd >= 1.0) return OR_INVALID_ARG;
	const uint64_t N = (uint64_t)1 << n;
	double cumulative = 0.0;
	for(uint64_t s = 0; s < N; ++s) {
		cumulative += a[2 * s] * a[2 * s] + a[2 * s + 1] * a[2 * s + 1];
		if(rnd <= cumulative) {
			*out = s;
			return OR_OK;
		}
	}
	return OR_RUNTIME;
}

/* Sequential logical amplitude sum, quantum_register.cpp:176-190 (no overlay). */
void or_dense_amplitude_sum(const double *a, unsigned n, double *re, double *im) {
	const uint64_t N = (uint64_t)1 << n;
	double sr = 0.0, si = 0.0;
	for(uint64_t s = 0; s < N; ++s) {
		sr += a[2 * s];
		si += a[2 * s + 1];
	}
	*re = sr;
	*im = si;
}

/* Generic k-qubit gate: validateGateTargets (validation.h:53-80),
 * makeGateBlockLayout (gate_block_apply.h:64-99), applyGateByBlocks
 * (gate_block_apply.h:103-213). */
int or_dense_gate(double *a, unsigned n, const double *g, const unsigned *qubits, unsigned k) {
	if(k > n) return OR_INVALID_ARG;
	{
		unsigned char seen[64] = {0};
		for(unsigned i = 0; i < k; ++i) {
			if(qubits[i] >= n) return OR_OUT_OF_RANGE;
			if(seen[qubits[i]]) return OR_INVALID_ARG;
			seen[qubits[i]] = 1;
		}
	}
	const uint64_t bs = (uint64_t)1 << k;
	const uint64_t nblocks = (uint64_t)1 << (n - k);
	uint64_t tmask[64];
	unsigned nontarget[64];
	unsigned nnt = 0;
	unsigned char is_t[64] = {0};
	for(unsigned i = 0; i < k; ++i) {
		const unsigned bit = n - qubits[i] - 1u;
		tmask[i] = (uint64_t)1 << bit;
		is_t[bit] = 1;
	}
	for(unsigned bit = 0; bit < n; ++bit)
		if(!is_t[bit]) nontarget[nnt++] = bit;
	uint64_t *offs = (uint64_t *)malloc(sizeof(uint64_t) * bs);
	double *loc = (double *)malloc(sizeof(double) * 2 * bs);
	uint64_t *idx = (uint64_t *)malloc(sizeof(uint64_t) * bs);
	if(!offs || !loc || !idx) {
		free(offs); free(loc); free(idx);
		return OR_NOMEM;
	}
	for(uint64_t j = 0; j < bs; ++j) {
		uint64_t off = 0;
		for(unsigned b = 0; b < k; ++b)
			if((j >> (k - b - 1u)) & 1u) off |= tmask[b];
		offs[j] = off;
	}
	for(uint64_t blk = 0; blk < nblocks; ++blk) {
		uint64_t base = 0;
		for(unsigned i = 0; i < nnt; ++i) base |= ((blk >> i) & 1u) << nontarget[i];
		if(k == 1) {
			const uint64_t s0 = base, s1 = base | tmask[0];
			const double a0r = a[2 * s0], a0i = a[2 * s0 + 1];
			const double a1r = a[2 * s1], a1i = a[2 * s1 + 1];
			if(a0r == 0.0 && a0i == 0.0 && a1r == 0.0 && a1i == 0.0) continue;
			const double g00r = g[0], g00i = g[1], g01r = g[2], g01i = g[3];
			const double g10r = g[4], g10i = g[5], g11r = g[6], g11i = g[7];
			a[2 * s0] = g00r * a0r - g00i * a0i + g01r * a1r - g01i * a1i;
			a[2 * s0 + 1] = g00r * a0i + g00i * a0r + g01r * a1i + g01i * a1r;
			a[2 * s1] = g10r * a0r - g10i * a0i + g11r * a1r - g11i * a1i;
			a[2 * s1 + 1] = g10r * a0i + g10i * a0r + g11r * a1i + g11i * a1r;
			continue;
		}
		int nonzero = 0;
		for(uint64_t j = 0; j < bs; ++j) {
			const uint64_t s = base | offs[j];
			idx[j] = s;
			loc[2 * j] = a[2 * s];
			loc[2 * j + 1] = a[2 * s + 1];
			if(loc[2 * j] != 0.0 || loc[2 * j + 1] != 0.0) nonzero = 1;
		}
		if(!nonzero) continue;
		for(uint64_t row = 0; row < bs; ++row) {
			double nr = 0.0, ni = 0.0;
			const double *grow = g + 2 * row * bs;
			for(uint64_t col = 0; col < bs; ++col) {
				const double gr = grow[2 * col], gi = grow[2 * col + 1];
				const double ar = loc[2 * col], ai = loc[2 * col + 1];
				nr += gr * ar - gi * ai;
				ni += gr * ai + gi * ar;
			}
			a[2 * idx[row]] = nr;
			a[2 * idx[row] + 1] = ni;
		}
	}
	free(offs); free(loc); free(idx);
	return OR_OK;
}

/* ---------------------------------------------------------------------- */
/* Register semantics, quantum_register.cpp                               */
/* ---------------------------------------------------------------------- */

static int reg_alloc(or_reg *r, unsigned n) {
	if(n > 40) return OR_INVALID_ARG;
	r->n = n;
	r->N = (uint64_t)1 << n;
	r->a = (double *)calloc((size_t)(2 * r->N), sizeof(double));
	if(!r->a) return OR_NOMEM;
	r->has_sum = 0;
	r->sum_re = r->sum_im = 0.0;
	r->overlay = 0;
	r->scale_re = 1.0; r->scale_im = 0.0;
	r->bias_re = 0.0; r->bias_im = 0.0;
	return OR_OK;
}

/* resetAffineOverlay, quantum_register.cpp:152-157. */
static void reset_overlay(or_reg *r) {
	r->scale_re = 1.0; r->scale_im = 0.0;
	r->bias_re = 0.0; r->bias_im = 0.0;
	r->overlay = 0;
	r->has_sum = 0;
}

/* applyAffineOverlay, quantum_register.cpp:160-165. */
static void apply_overlay(const or_reg *r, double re, double im, double *ore, double *oim) {
	if(!r->overlay) { *ore = re; *oim = im; return; }
	const double mr = r->scale_re * re - r->scale_im * im;
	const double mi = r->scale_re * im + r->scale_im * re;
	*ore = mr + r->bias_re;
	*oim = mi + r->bias_im;
}

/* removeAffineOverlay + divideAmplitude, quantum_register.cpp:44-53,168-173. */
static int remove_overlay(const or_reg *r, double re, double im, double *ore, double *oim) {
	if(!r->overlay) { *ore = re; *oim = im; return OR_OK; }
	const double nr = re - r->bias_re;
	const double ni = im - r->bias_im;
	const double dr = r->scale_re, di = r->scale_im;
	const double d = dr * dr + di * di;
	if(d == 0.0) return OR_LOGIC;
	*ore = (nr * dr + ni * di) / d;
	*oim = (ni * dr - nr * di) / d;
	return OR_OK;
}

/* flushAffineOverlay, quantum_register.cpp:223-231. */
static void flush_overlay(or_reg *r) {
	if(!r->overlay) return;
	const int had = r->has_sum;
	const double sr = r->sum_re, si = r->sum_im;
	or_dense_affine(r->a, r->n, r->scale_re, r->scale_im, r->bias_re, r->bias_im);
	reset_overlay(r);
	r->has_sum = had;
	r->sum_re = sr;
	r->sum_im = si;
}

/* logicalAmplitudeSum, quantum_register.cpp:176-190. */
static void logical_sum(or_reg *r, double *re, double *im) {
	if(r->has_sum) { *re = r->sum_re; *im = r->sum_im; return; }
	double sr = 0.0, si = 0.0;
	for(uint64_t s = 0; s < r->N; ++s) {
		double lr, li;
		apply_overlay(r, r->a[2 * s], r->a[2 * s + 1], &lr, &li);
		sr += lr;
		si += li;
	}
	r->has_sum = 1;
	r->sum_re = sr;
	r->sum_im = si;
	*re = sr;
	*im = si;
}

/* QuantumRegister(n, s, amp, cfg) -> initBasis, quantum_register.cpp:84-96; dense_state_backend.cpp:84-90. */
int or_reg_init_basis(or_reg *r, unsigned n, uint64_t s, double re, double im) {
	int rc = reg_alloc(r, n);
	if(rc) return rc;
	if(s >= r->N) { or_reg_free(r); return OR_OUT_OF_RANGE; }
	r->a[2 * s] = re;
	r->a[2 * s + 1] = im;
	return OR_OK;
}

static int cmp_u64(const void *x, const void *y) {
	const uint64_t a = *(const uint64_t *)x, b = *(const uint64_t *)y;
	return a < b ? -1 : (a > b ? 1 : 0);
}

/* initUniformSuperposition, quantum_register.cpp:331-341; dense_state_backend.cpp:92-115. */
int or_reg_init_uniform(or_reg *r, unsigned n, const uint64_t *states, size_t count) {
	int rc = reg_alloc(r, n);
	if(rc) return rc;
	if(count == 0) { or_reg_free(r); return OR_INVALID_ARG; }
	uint64_t *sel = (uint64_t *)malloc(sizeof(uint64_t) * count);
	if(!sel) { or_reg_free(r); return OR_NOMEM; }
	for(size_t i = 0; i < count; ++i) {
		if(states[i] >= r->N) { free(sel); or_reg_free(r); return OR_OUT_OF_RANGE; }
		sel[i] = states[i];
	}
	qsort(sel, count, sizeof(uint64_t), cmp_u64);
	size_t u = 0;
	for(size_t i = 0; i < count; ++i)
		if(u == 0 || sel[u - 1] != sel[i]) sel[u++] = sel[i];
	const double amp = 1.0 / sqrt((double)u);
	for(size_t i = 0; i < u; ++i) {
		r->a[2 * sel[i]] = amp;
		r->a[2 * sel[i] + 1] = 0.0;
	}
	free(sel);
	return OR_OK;
}

/* QuantumRegister(n, amplitudes, cfg) -> loadAmplitudes, quantum_register.cpp:98-103. */
int or_reg_load(or_reg *r, unsigned n, const double *amps) {
	int rc = reg_alloc(r, n);
	if(rc) return rc;
	memcpy(r->a, amps, sizeof(double) * 2 * r->N);
	return OR_OK;
}

void or_reg_free(or_reg *r) {
	free(r->a);
	r->a = NULL;
}

/* Copy constructor, quantum_register.cpp:106-119. */
int or_reg_copy(or_reg *dst, const or_reg *src) {
	*dst = *src;
	dst->a = (double *)malloc(sizeof(double) * 2 * src->N);
	if(!dst->a) return OR_NOMEM;
	memcpy(dst->a, src->a, sizeof(double) * 2 * src->N);
	return OR_OK;
}

/* amplitude, quantum_register.cpp:249-253. */
int or_reg_amplitude(const or_reg *r, uint64_t s, double *re, double *im) {
	if(s >= r->N) return OR_OUT_OF_RANGE;
	apply_overlay(r, r->a[2 * s], r->a[2 * s + 1], re, im);
	return OR_OK;
}

/* setAmplitude, quantum_register.cpp:313-318. */
int or_reg_set_amplitude(or_reg *r, uint64_t s, double re, double im) {
	if(s >= r->N) return OR_OUT_OF_RANGE;
	double br, bi;
	int rc = remove_overlay(r, re, im, &br, &bi);
	if(rc) return rc;
	r->a[2 * s] = br;
	r->a[2 * s + 1] = bi;
	r->has_sum = 0;
	return OR_OK;
}

/* amplitudes() / snapshotLogicalAmplitudes, quantum_register.cpp:213-220,256-259. */
int or_reg_export(const or_reg *r, double *out) {
	for(uint64_t s = 0; s < r->N; ++s) apply_overlay(r, r->a[2 * s], r->a[2 * s + 1], &out[2 * s], &out[2 * s + 1]);
	return OR_OK;
}

/* totalProbability, quantum_register.cpp:269-282. */
double or_reg_total_probability(const or_reg *r) {
	if(!r->overlay) return or_dense_total_probability(r->a, r->n);
	double total = 0.0;
	for(uint64_t s = 0; s < r->N; ++s) {
		double lr, li;
		apply_overlay(r, r->a[2 * s], r->a[2 * s + 1], &lr, &li);
		total += lr * lr + li * li;
	}
	return total;
}

/* measure, quantum_register.cpp:284-310 (the random draw is the caller's). */
int or_reg_measure(const or_reg *r, double rnd, uint64_t *out) {
	if(!r->overlay) return or_dense_sample(r->a, r->n, rnd, out);
	double cumulative = 0.0;
	for(uint64_t s = 0; s < r->N; ++s) {
		double lr, li;
		apply_overlay(r, r->a[2 * s], r->a[2 * s + 1], &lr, &li);
		cumulative += lr * lr + li * li;
		if(rnd <= cumulative) {
			*out = s;
			return OR_OK;
		}
	}
	return OR_RUNTIME;
}

/* applyInversionAboutMean(mean) (lazy, quantum_register.cpp:433-444) and
 * applyInversionAboutMeanMaterialized(mean) (quantum_register.cpp:457-467). */
int or_reg_inversion_mean(or_reg *r, double mre, double mim, int materialized) {
	if(r->has_sum) {
		r->sum_re = 2.0 * mre * (double)r->N - r->sum_re;
		r->sum_im = 2.0 * mim * (double)r->N - r->sum_im;
	}
	if(materialized) {
		if(r->overlay) flush_overlay(r);
		or_dense_inversion_mean(r->a, r->n, mre, mim);
		return OR_OK;
	}
	const double sr = r->overlay ? r->scale_re : 1.0;
	const double si = r->overlay ? r->scale_im : 0.0;
	const double br = r->overlay ? r->bias_re : 0.0;
	const double bi = r->overlay ? r->bias_im : 0.0;
	r->scale_re = -sr;
	r->scale_im = -si;
	r->bias_re = mre * 2.0 - br;
	r->bias_im = mim * 2.0 - bi;
	r->overlay = 1;
	return OR_OK;
}

static int check_qubit(const or_reg *r, unsigned q) { return q < r->n ? OR_OK : OR_OUT_OF_RANGE; }

/* Register-level dispatch of one circuit operation: executeOperation
 * (simulator.cpp:17-44) over the QuantumRegister methods
 * (quantum_register.cpp:394-527). */
int or_reg_apply(or_reg *r, const or_op *op) {
	int rc;
	switch(op->kind) {
		case OR_OP_H:
			if((rc = check_qubit(r, op->q0))) return rc;
			flush_overlay(r);
			or_dense_h(r->a, r->n, op->q0);
			r->has_sum = 0;
			return OR_OK;
		case OR_OP_X:
			if((rc = check_qubit(r, op->q0))) return rc;
			flush_overlay(r);
			or_dense_x(r->a, r->n, op->q0);
			r->has_sum = 0;
			return OR_OK;
		case OR_OP_CNOT:
		case OR_OP_CPHASE:
			if((rc = check_qubit(r, op->q0))) return rc;
			if((rc = check_qubit(r, op->q1))) return rc;
			if(op->q0 == op->q1) return OR_INVALID_ARG;
			flush_overlay(r);
			if(op->kind == OR_OP_CNOT) or_dense_cnot(r->a, r->n, op->q0, op->q1);
			else or_dense_cphase(r->a, r->n, op->q0, op->q1, op->theta);
			r->has_sum = 0;
			return OR_OK;
		case OR_OP_SWAP: {
			/* applySwap = CNOT(a,b), CNOT(b,a), CNOT(a,b), quantum_register.cpp:518-527. */
			if((rc = check_qubit(r, op->q0))) return rc;
			if((rc = check_qubit(r, op->q1))) return rc;
			if(op->q0 == op->q1) return OR_INVALID_ARG;
			or_op c = *op;
			c.kind = OR_OP_CNOT;
			if((rc = or_reg_apply(r, &c))) return rc;
			c.q0 = op->q1; c.q1 = op->q0;
			if((rc = or_reg_apply(r, &c))) return rc;
			c.q0 = op->q0; c.q1 = op->q1;
			return or_reg_apply(r, &c);
		}
		case OR_OP_GATE:
			if(op->k > r->n) return OR_INVALID_ARG;
			{
				unsigned char seen[64] = {0};
				for(unsigned i = 0; i < op->k; ++i) {
					if(op->qubits[i] >= r->n) return OR_OUT_OF_RANGE;
					if(seen[op->qubits[i]]) return OR_INVALID_ARG;
					seen[op->qubits[i]] = 1;
				}
			}
			flush_overlay(r);
			rc = or_dense_gate(r->a, r->n, op->matrix, op->qubits, op->k);
			r->has_sum = 0;
			return rc;
		case OR_OP_PHASE_FLIP: {
			/* applyPhaseFlipBasisState, quantum_register.cpp:405-420. */
			const uint64_t s = op->state;
			if(s >= r->N) return OR_OUT_OF_RANGE;
			if(r->has_sum || r->overlay) {
				double lr, li;
				or_reg_amplitude(r, s, &lr, &li);
				if(r->has_sum) {
					r->sum_re -= 2.0 * lr;
					r->sum_im -= 2.0 * li;
				}
				if(r->overlay) {
					double br, bi;
					if((rc = remove_overlay(r, -lr, -li, &br, &bi))) return rc;
					r->a[2 * s] = br;
					r->a[2 * s + 1] = bi;
					return OR_OK;
				}
			}
			or_dense_phase_flip(r->a, s);
			return OR_OK;
		}
		case OR_OP_INVERSION: {
			/* applyInversionAboutMean[Materialized](), quantum_register.cpp:423-431,447-455. */
			double sr, si;
			logical_sum(r, &sr, &si);
			return or_reg_inversion_mean(r, sr / (double)r->N, si / (double)r->N, op->materialized);
		}
		default:
			return OR_INVALID_ARG;
	}
}

/* Simulator::run op loop, simulator.cpp:54-96 (timing and traces omitted). */
int or_reg_run(or_reg *r, const or_op *ops, size_t nops) {
	for(size_t i = 0; i < nops; ++i) {
		int rc = or_reg_apply(r, &ops[i]);
		if(rc) return rc;
	}
	return OR_OK;
}

/* ---------------------------------------------------------------------- */
/* Circuits, circuit.cpp                                                  */
/* ---------------------------------------------------------------------- */

size_t or_qft_op_count(unsigned n) { return (size_t)n + (size_t)n * (n - 1) / 2 + n / 2; }

/* appendQft, circuit.cpp:87-100. */
size_t or_build_qft(unsigned n, or_op *ops) {
	size_t k = 0;
	for(unsigned t = 0; t < n; ++t) {
		memset(&ops[k], 0, sizeof(or_op));
		ops[k].kind = OR_OP_H;
		ops[k].q0 = t;
		++k;
		for(unsigned c = t + 1u; c < n; ++c) {
			const unsigned d = c - t;
			memset(&ops[k], 0, sizeof(or_op));
			ops[k].kind = OR_OP_CPHASE;
			ops[k].q0 = c;
			ops[k].q1 = t;
			ops[k].theta = OR_PI / (double)((uint64_t)1 << d);
			++k;
		}
	}
	for(unsigned l = 0; l < n / 2u; ++l) {
		memset(&ops[k], 0, sizeof(or_op));
		ops[k].kind = OR_OP_SWAP;
		ops[k].q0 = l;
		ops[k].q1 = n - l - 1u;
		++k;
	}
	return k;
}

/* groverIterationCount, circuit.cpp:108-116. */
unsigned or_grover_iterations(uint64_t state_count, size_t marked_count) {
	if(marked_count == 0) return 0;
	const double ideal = (OR_PI / 4.0) * sqrt((double)state_count / (double)marked_count);
	return (unsigned)floor(ideal);
}

/* appendGrover, circuit.cpp:118-141.  Returns the op count, or a negative
 * error code (-OR_INVALID_ARG) where the reference throws. */
long or_build_grover(unsigned n, const uint64_t *marked, size_t count, int materialized,
                     uint64_t *sorted_out, size_t *unique_out, or_op *ops) {
	if(count == 0) return -OR_INVALID_ARG;
	uint64_t *sel = sorted_out;
	memcpy(sel, marked, sizeof(uint64_t) * count);
	qsort(sel, count, sizeof(uint64_t), cmp_u64);
	size_t u = 0;
	for(size_t i = 0; i < count; ++i)
		if(u == 0 || sel[u - 1] != sel[i]) sel[u++] = sel[i];
	*unique_out = u;
	const uint64_t N = (uint64_t)1 << n;
	const unsigned iters = or_grover_iterations(N, u);
	long k = 0;
	for(unsigned q = 0; q < n; ++q) {
		if(ops) {
			memset(&ops[k], 0, sizeof(or_op));
			ops[k].kind = OR_OP_H;
			ops[k].q0 = q;
		}
		++k;
	}
	for(unsigned it = 0; it < iters; ++it) {
		for(size_t i = 0; i < u; ++i) {
			if(sel[i] >= N) return -OR_INVALID_ARG;
			if(ops) {
				memset(&ops[k], 0, sizeof(or_op));
				ops[k].kind = OR_OP_PHASE_FLIP;
				ops[k].state = sel[i];
			}
			++k;
		}
		if(ops) {
			memset(&ops[k], 0, sizeof(or_op));
			ops[k].kind = OR_OP_INVERSION;
			ops[k].materialized = materialized;
		}
		++k;
	}
	return k;
}

/* ---------------------------------------------------------------------- */
/* RNG: std::mt19937 (published MT19937 algorithm) and libstdc++          */
/* generate_canonical<double, 53> as used by                              */
/* uniform_real_distribution<double> (random.h:32-58, random.cpp:6-16).   */
/* ---------------------------------------------------------------------- */

void or_mt_seed(or_mt19937 *g, uint32_t seed) {
	g->mt[0] = seed;
	for(int i = 1; i < 624; ++i) g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
	g->idx = 624;
}

static void mt_twist(or_mt19937 *g) {
	for(int i = 0; i < 624; ++i) {
		const uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
		uint32_t v = g->mt[(i + 397) % 624] ^ (y >> 1);
		if(y & 1u) v ^= 0x9908b0dfu;
		g->mt[i] = v;
	}
	g->idx = 0;
}

uint32_t or_mt_next(or_mt19937 *g) {
	if(g->idx >= 624) mt_twist(g);
	uint32_t y = g->mt[g->idx++];
	y ^= y >> 11;
	y ^= (y << 7) & 0x9d2c5680u;
	y ^= (y << 15) & 0xefc60000u;
	y ^= y >> 18;
	return y;
}

/* generate_canonical<double,53>: two 32-bit draws, sum = g1 + g2*2^32 in
 * double, divided by 2^64, clamped below 1. */
double or_mt_canonical(or_mt19937 *g) {
	double sum = 0.0;
	double tmp = 1.0;
	for(int k = 0; k < 2; ++k) {
		sum += (double)or_mt_next(g) * tmp;
		tmp *= 4294967296.0;
	}
	double ret = sum / tmp;
	if(ret >= 1.0) ret = nextafter(1.0, 0.0);
	return ret;
}

/* QuantumState::randomPhase, quantum_state.cpp:264-277 (= buildRandomPhaseInput, qftG.cpp:70-81). */
void or_random_phase(unsigned n, uint32_t seed, double *out) {
	const uint64_t N = (uint64_t)1 << n;
	or_mt19937 g;
	or_mt_seed(&g, seed);
	const double width = 2.0 * acos(-1.0) - 0.0;
	const double norm = 1.0 / sqrt((double)N);
	for(uint64_t s = 0; s < N; ++s) {
		const double phase = or_mt_canonical(&g) * width + 0.0;
		out[2 * s] = norm * cos(phase);
		out[2 * s + 1] = norm * sin(phase);
	}
}
