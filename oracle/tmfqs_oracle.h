/*
 * CPU oracle for the dense state-vector path of TMFQS (test infrastructure).
 *
 * This is a plain-C restatement of the reference's Dense backend, register
 * overlay logic, circuit builders and RNG.  It exists only so that tests,
 * the smoke check and the CPU-baseline leg of the bench can check the CUDA
 * path against it; nothing in the product links or calls it.
 *
 * Arithmetic is written so that every floating-point operation is one IEEE
 * double operation in the same order as the reference C++ (compiled without
 * FMA contraction: -O3, no -march), so results are bit-identical to the
 * reference on the same glibc.  Parity of this restatement is pinned against
 * the reference itself, compiled from its sources into oracle/_ref, by
 * tests/test_oracle_pinned.py, and against the golden values in
 * tests/golden/.
 *
 * Qubit q maps to bit (n-1-q) of the state index (qubit 0 = most
 * significant), as in include/tmfqs/core/types.h:12-13 of the reference.
 */
#ifndef TMFQS_ORACLE_H
#define TMFQS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Operation kinds: the circuit::Operation variant, circuit.h:16-61. */
enum {
	OR_OP_H = 0,
	OR_OP_X = 1,
	OR_OP_CNOT = 2,
	OR_OP_CPHASE = 3,
	OR_OP_SWAP = 4,
	OR_OP_GATE = 5,
	OR_OP_PHASE_FLIP = 6,
	OR_OP_INVERSION = 7
};

typedef struct {
	int kind;
	unsigned q0;          /* target (H, X) / control (CNOT, CPHASE) / first (SWAP) */
	unsigned q1;          /* target (CNOT, CPHASE) / second (SWAP) */
	double theta;         /* CPHASE angle */
	uint64_t state;       /* PHASE_FLIP basis state */
	int materialized;     /* INVERSION: materialised (1) or lazy overlay (0) */
	const double *matrix; /* GATE: row-major 2^k x 2^k interleaved complex */
	const unsigned *qubits; /* GATE: target list, MSB-first block order */
	unsigned k;           /* GATE: number of targets */
} or_op;

/* Register: dense amplitudes plus the lazy affine overlay and the cached
 * logical amplitude sum of QuantumRegister (quantum_register.h:207-224). */
typedef struct {
	unsigned n;
	uint64_t N;
	double *a;            /* interleaved [re0, im0, re1, im1, ...], 2N doubles */
	int has_sum;
	double sum_re, sum_im;
	int overlay;
	double scale_re, scale_im, bias_re, bias_im;
} or_reg;

/* Error codes (mirrors of the reference's exception classes). */
enum {
	OR_OK = 0,
	OR_OUT_OF_RANGE = 1,   /* std::out_of_range */
	OR_INVALID_ARG = 2,    /* std::invalid_argument */
	OR_LOGIC = 3,          /* std::logic_error */
	OR_RUNTIME = 4,        /* std::runtime_error */
	OR_NOMEM = 5
};

/* ---- backend-level kernels on a raw interleaved buffer ---------------- */
void or_dense_h(double *a, unsigned n, unsigned q);
void or_dense_x(double *a, unsigned n, unsigned q);
void or_dense_cnot(double *a, unsigned n, unsigned c, unsigned t);
void or_dense_cphase(double *a, unsigned n, unsigned c, unsigned t, double theta);
void or_dense_phase_flip(double *a, uint64_t s);
void or_dense_inversion_mean(double *a, unsigned n, double mre, double mim);
void or_dense_inversion(double *a, unsigned n);
void or_dense_affine(double *a, unsigned n, double sre, double sim, double bre, double bim);
double or_dense_total_probability(const double *a, unsigned n);
int or_dense_sample(const double *a, unsigned n, double rnd, uint64_t *out);
int or_dense_gate(double *a, unsigned n, const double *matrix, const unsigned *qubits, unsigned k);
void or_dense_amplitude_sum(const double *a, unsigned n, double *re, double *im);

/* ---- register-level semantics (overlay + cached sum) ------------------ */
int or_reg_init_basis(or_reg *r, unsigned n, uint64_t s, double re, double im);
int or_reg_init_uniform(or_reg *r, unsigned n, const uint64_t *states, size_t count);
int or_reg_load(or_reg *r, unsigned n, const double *amps);
void or_reg_free(or_reg *r);
int or_reg_copy(or_reg *dst, const or_reg *src);
int or_reg_apply(or_reg *r, const or_op *op);
int or_reg_run(or_reg *r, const or_op *ops, size_t nops);
int or_reg_amplitude(const or_reg *r, uint64_t s, double *re, double *im);
int or_reg_set_amplitude(or_reg *r, uint64_t s, double re, double im);
int or_reg_export(const or_reg *r, double *out);
double or_reg_total_probability(const or_reg *r);
int or_reg_measure(const or_reg *r, double rnd, uint64_t *out);
int or_reg_inversion_mean(or_reg *r, double mre, double mim, int materialized);

/* ---- circuits --------------------------------------------------------- */
size_t or_qft_op_count(unsigned n);
size_t or_build_qft(unsigned n, or_op *ops);
unsigned or_grover_iterations(uint64_t state_count, size_t marked_count);
/* Writes the deduplicated sorted marked list into `sorted_out` (capacity
 * count) and returns the op count; ops may be NULL to query the count. */
long or_build_grover(unsigned n, const uint64_t *marked, size_t count, int materialized,
                     uint64_t *sorted_out, size_t *unique_out, or_op *ops);

/* ---- RNG -------------------------------------------------------------- */
typedef struct {
	uint32_t mt[624];
	int idx;
} or_mt19937;
void or_mt_seed(or_mt19937 *g, uint32_t seed);
uint32_t or_mt_next(or_mt19937 *g);
double or_mt_canonical(or_mt19937 *g);
void or_random_phase(unsigned n, uint32_t seed, double *out);

#ifdef __cplusplus
}
#endif

#endif
