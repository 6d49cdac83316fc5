/*
 * nemo_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity checker).
 *
 * A plain-C restatement of the NeMo 0.7.2 reference CPU backend.  Every
 * function cites the reference file:line it restates.  Build with
 * -O2 -ffp-contract=off and no -march (the reference's x86-64 build has no
 * FMA contraction; see oracle/Makefile).  OpenMP parallelises exactly the
 * loops the reference parallelises (neuron update and current conversion);
 * spike delivery and STDP accumulation stay serial as in the reference.
 *
 * Deliberately reproduced x86-64 behaviours of the reference:
 *  - variable 64-bit shifts use the low 6 bits of the count, so a network
 *    whose maximum delay is exactly 64 delivers no spikes
 *    (src/nemo/cpu/Simulation.cpp:263);
 *  - signed int32 accumulator/weight arithmetic wraps;
 *  - float->unsigned conversion goes through a 64-bit truncation.
 */
#include "nemo_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* src/nemo/types.h:31-61 */
enum {
	NEMO_OK = 0,
	NEMO_API_UNSUPPORTED = 5,
	NEMO_INVALID_INPUT = 6,
	NEMO_BUFFER_OVERFLOW = 7,
	NEMO_LOGIC_ERROR = 9,
	NEMO_ALLOCATION_ERROR = 10,
	NEMO_UNKNOWN_ERROR = 14
};

#define FBITS 20 /* src/nemo/ConfigurationImpl.cpp:22 */
#define MAX_HISTORY 64 /* src/nemo/StdpFunction.cpp:151 */

static char g_err[512];

static int fail(int code, const char* fmt, ...)
{
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(g_err, sizeof g_err, fmt, ap);
	va_end(ap);
	return code;
}

const char* nemo_oracle_strerror(void) { return g_err; }

/* --------------------------------------------------------------------- */
/* x86-64 shift semantics                                                 */

static inline uint64_t shl64(uint64_t x, unsigned s) { return x << (s & 63); }
static inline uint64_t shr64(uint64_t x, unsigned s) { return x >> (s & 63); }

/* --------------------------------------------------------------------- */
/* Fixed point: src/nemo/fixedpoint.cpp:17-49, src/nemo/fixedpoint.hpp:41-50 */

static int fx_toFix(float f, int32_t* out)
{
	/* fixedpoint.cpp:20: abs(int(f)) >= 1 << (31 - fbits) throws */
	int i = (int) f;
	if(abs(i) >= (1 << (31 - FBITS))) {
		return fail(NEMO_UNKNOWN_ERROR,
				"Fixed-point overflow. Value %g does not fit into fixed-point format Q%u.%u",
				(double) f, 31 - FBITS, FBITS);
	}
	*out = (int32_t) (f * (float) (1 << FBITS));
	return NEMO_OK;
}

static inline float fx_toFloat(int32_t v) { return (float) v / (float) (1 << FBITS); }

static inline float wfx_toFloat(int64_t v)
{
	/* saturation is on in the reference build (src/nemo/CMakeLists.txt:1) */
	if(v > (int64_t) INT32_MAX) v = INT32_MAX;
	if(v < (int64_t) INT32_MIN) v = INT32_MIN;
	return (float) v / (float) (1 << FBITS);
}

static inline int32_t fx_mul(int32_t a, int32_t b)
{
	int64_t r = (int64_t) a * (int64_t) b;
	return (int32_t) (r >> FBITS);
}

static inline int32_t wrap_add32(int32_t a, int32_t b)
{
	return (int32_t) ((uint32_t) a + (uint32_t) b);
}

/* --------------------------------------------------------------------- */
/* RNG: src/nemo/RNG.cpp:9-63                                             */

unsigned nemo_oracle_urand(unsigned s[4])
{
	unsigned t = (s[0] ^ (s[0] << 11));
	s[0] = s[1];
	s[1] = s[2];
	s[2] = s[3];
	s[3] = (s[3] ^ (s[3] >> 19)) ^ (t ^ (t >> 8));
	return s[3];
}

float nemo_oracle_nrand(unsigned s[4])
{
	/* RNG.cpp:27-32, evaluated in statement order */
	float a = nemo_oracle_urand(s) * 1.4629180792671596810513378043098e-9f;
	float b = nemo_oracle_urand(s) * 0.00000000023283064365386962890625f;
	float r = sqrtf(-2 * logf(1 - b));
	return sinf(a) * r;
}

/* mt19937, identical to boost::mt19937 / std::mt19937 with default seed 5489 */
typedef struct { uint32_t mt[624]; int i; } mt19937;

static void mt_seed(mt19937* g, uint32_t seed)
{
	g->mt[0] = seed;
	for(int i = 1; i < 624; ++i) {
		g->mt[i] = 1812433253u * (g->mt[i-1] ^ (g->mt[i-1] >> 30)) + (uint32_t) i;
	}
	g->i = 624;
}

static uint32_t mt_next(mt19937* g)
{
	if(g->i >= 624) {
		for(int k = 0; k < 624; ++k) {
			uint32_t y = (g->mt[k] & 0x80000000u) | (g->mt[(k+1) % 624] & 0x7fffffffu);
			g->mt[k] = g->mt[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
		}
		g->i = 0;
	}
	uint32_t y = g->mt[g->i++];
	y ^= (y >> 11);
	y ^= (y << 7) & 0x9d2c5680u;
	y ^= (y << 15) & 0xefc60000u;
	y ^= (y >> 18);
	return y;
}

/* boost::uniform_int<unsigned long>(0, 0x7fffffff) over a 32-bit engine:
 * bucket size 2, i.e. x >> 1 (Boost >= 1.47 uniform_int_distribution) */
void nemo_oracle_seed_states(unsigned first, unsigned count, unsigned* out)
{
	/* RNG.cpp:38-63: a fresh default-seeded stream, 4*first draws
	 * discarded, then 4 words per neuron */
	mt19937 g;
	mt_seed(&g, 5489u);
	for(unsigned i = 0; i < 4u * first; ++i) {
		(void) mt_next(&g);
	}
	for(unsigned n = 0; n < count; ++n) {
		for(unsigned p = 0; p < 4; ++p) {
			out[4*n + p] = mt_next(&g) >> 1;
		}
	}
}

/* --------------------------------------------------------------------- */
/* Small open-addressing hash map u32 -> u64                              */

typedef struct { uint32_t* keys; uint64_t* vals; uint8_t* used; size_t cap, n; } hmap;

static uint32_t hkey(uint32_t k) { k ^= k >> 16; k *= 0x7feb352du; k ^= k >> 15; k *= 0x846ca68bu; k ^= k >> 16; return k; }

static void hmap_free(hmap* m) { free(m->keys); free(m->vals); free(m->used); memset(m, 0, sizeof *m); }

static int hmap_grow(hmap* m)
{
	size_t ncap = m->cap ? m->cap * 2 : 1024;
	hmap nm = { calloc(ncap, 4), calloc(ncap, 8), calloc(ncap, 1), ncap, 0 };
	if(!nm.keys || !nm.vals || !nm.used) { hmap_free(&nm); return -1; }
	for(size_t i = 0; i < m->cap; ++i) {
		if(m->used[i]) {
			size_t j = hkey(m->keys[i]) & (ncap - 1);
			while(nm.used[j]) j = (j + 1) & (ncap - 1);
			nm.used[j] = 1; nm.keys[j] = m->keys[i]; nm.vals[j] = m->vals[i]; nm.n++;
		}
	}
	hmap_free(m);
	*m = nm;
	return 0;
}

static uint64_t* hmap_find(const hmap* m, uint32_t k)
{
	if(!m->cap) return NULL;
	size_t j = hkey(k) & (m->cap - 1);
	while(m->used[j]) {
		if(m->keys[j] == k) return &m->vals[j];
		j = (j + 1) & (m->cap - 1);
	}
	return NULL;
}

/* returns 1 if inserted, 0 if present (value untouched), -1 on alloc failure */
static int hmap_insert(hmap* m, uint32_t k, uint64_t v, uint64_t** slot)
{
	if((m->n + 1) * 2 > m->cap && hmap_grow(m)) return -1;
	size_t j = hkey(k) & (m->cap - 1);
	while(m->used[j]) {
		if(m->keys[j] == k) { if(slot) *slot = &m->vals[j]; return 0; }
		j = (j + 1) & (m->cap - 1);
	}
	m->used[j] = 1; m->keys[j] = k; m->vals[j] = v; m->n++;
	if(slot) *slot = &m->vals[j];
	return 1;
}

/* --------------------------------------------------------------------- */
/* Neuron types: .ini descriptors src/nemo/plugins/<Type>.ini and index   */
/* headers src/nemo/plugins/Izhikevich.h, IF_curr_exp.h                   */

enum { KIND_IZHIKEVICH, KIND_IF_CURR_EXP, KIND_POISSON, KIND_INPUT, KIND_IZHIKEVICH_RS, KIND_KURAMOTO };

/* history: state history length; rcm: needs the reverse matrix of all
 * synapses (sources, delays, weights) */
typedef struct { const char* name; int kind; unsigned nparam, nstate, mpot, history; int rcm; } type_desc;

static const type_desc TYPES[] = {
	{ "Izhikevich", KIND_IZHIKEVICH, 5, 2, 1, 1, 0 },    /* Izhikevich.ini:2-4 */
	{ "IF_curr_exp", KIND_IF_CURR_EXP, 9, 4, 0, 1, 0 },  /* IF_curr_exp.ini:14-24 */
	{ "PoissonSource", KIND_POISSON, 1, 0, 0, 1, 0 },    /* PoissonSource.ini:1-3 */
	{ "Input", KIND_INPUT, 0, 0, 0, 1, 0 },              /* Input.ini:1-3 */
	{ "IzhikevichRS", KIND_IZHIKEVICH_RS, 0, 2, 1, 1, 0 },  /* IzhikevichRS.ini:3-5 */
	{ "Kuramoto", KIND_KURAMOTO, 1, 1, 0, 32, 1 },       /* Kuramoto.ini:2-14 */
};
#define NTYPES_KNOWN (sizeof TYPES / sizeof TYPES[0])

typedef struct {
	const type_desc* desc;
	size_t n, cap;
	unsigned* gidx;
	float* args; /* n x (nparam + nstate), insertion order */
} neuron_coll;

typedef struct {
	unsigned* src; unsigned* tgt; unsigned* delay; float* weight; unsigned char* plastic;
	uint32_t* sid;     /* per-source synapse index (synapse id low word) */
	size_t n, cap;
} syn_store;

struct nemo_oracle_network {
	neuron_coll types[16];
	unsigned ntypes;
	hmap neurons;   /* gidx -> (type << 32) | index */
	hmap axons;     /* source gidx -> number of synapses */
	syn_store syn;
	unsigned maxDelay;
	int duplicate;
	unsigned dupIdx;
};

struct nemo_oracle_configuration {
	int stdp;
	float* pre; size_t npre;
	float* post; size_t npost;
	float minE, maxE, minI, maxI;
	int writeOnly;
};

/* --------------------------------------------------------------------- */
/* Configuration                                                          */

nemo_oracle_configuration* nemo_oracle_new_configuration(void)
{
	return calloc(1, sizeof(nemo_oracle_configuration));
}

void nemo_oracle_delete_configuration(nemo_oracle_configuration* c)
{
	if(c) { free(c->pre); free(c->post); free(c); }
}

/* StdpFunction ctor checks: src/nemo/StdpFunction.cpp:12-47 */
int nemo_oracle_set_stdp_function(nemo_oracle_configuration* c,
		const float* prefire, size_t npre, const float* postfire, size_t npost,
		float minE, float maxE, float minI, float maxI)
{
	if(maxI > 0.0f || minI > 0.0f)
		return fail(NEMO_INVALID_INPUT, "STDP function should not have positive limits for inhibitory synapses");
	if(maxE < 0.0f || minE < 0.0f)
		return fail(NEMO_INVALID_INPUT, "STDP function should not have negative limits for inhibitory synapses");
	if(maxE < minE)
		return fail(NEMO_INVALID_INPUT, "STDP should have maximum excitatory weight >= minimum excitatory weight");
	if(maxI > minI)
		return fail(NEMO_INVALID_INPUT, "STDP should have abs(maximum inhibitory weight) >= abs(minimum inhibitory weight)");
	if(npre + npost > MAX_HISTORY)
		return fail(NEMO_INVALID_INPUT, "size of STDP window too large");
	free(c->pre); free(c->post);
	c->pre = malloc((npre ? npre : 1) * sizeof(float));
	c->post = malloc((npost ? npost : 1) * sizeof(float));
	if(npre) memcpy(c->pre, prefire, npre * sizeof(float));
	if(npost) memcpy(c->post, postfire, npost * sizeof(float));
	c->npre = npre; c->npost = npost;
	c->minE = minE; c->maxE = maxE; c->minI = minI; c->maxI = maxI;
	c->stdp = 1;
	return NEMO_OK;
}

int nemo_oracle_set_write_only_synapses(nemo_oracle_configuration* c)
{
	c->writeOnly = 1;
	return NEMO_OK;
}

/* --------------------------------------------------------------------- */
/* Network: src/nemo/NetworkImpl.cpp, src/nemo/Neurons.cpp, src/nemo/Axon.cpp */

nemo_oracle_network* nemo_oracle_new_network(void)
{
	return calloc(1, sizeof(nemo_oracle_network));
}

void nemo_oracle_delete_network(nemo_oracle_network* net)
{
	if(!net) return;
	for(unsigned t = 0; t < net->ntypes; ++t) {
		free(net->types[t].gidx);
		free(net->types[t].args);
	}
	hmap_free(&net->neurons);
	hmap_free(&net->axons);
	free(net->syn.src); free(net->syn.tgt); free(net->syn.delay);
	free(net->syn.weight); free(net->syn.plastic); free(net->syn.sid);
	free(net);
}

/* NetworkImpl::addNeuronType, NetworkImpl.cpp:37-48 */
int nemo_oracle_add_neuron_type(nemo_oracle_network* net, const char* name, unsigned* type)
{
	for(unsigned t = 0; t < net->ntypes; ++t) {
		if(strcmp(net->types[t].desc->name, name) == 0) { *type = t; return NEMO_OK; }
	}
	const type_desc* d = NULL;
	for(unsigned i = 0; i < NTYPES_KNOWN; ++i) {
		if(strcmp(TYPES[i].name, name) == 0) d = &TYPES[i];
	}
	if(!d) return fail(NEMO_INVALID_INPUT, "Could not find neuron type configuration file %s.ini", name);
	if(net->ntypes >= 16) return fail(NEMO_API_UNSUPPORTED, "too many neuron types");
	memset(&net->types[net->ntypes], 0, sizeof(neuron_coll));
	net->types[net->ntypes].desc = d;
	*type = net->ntypes++;
	return NEMO_OK;
}

/* NetworkImpl::addNeuron (NetworkImpl.cpp:84-92) -> Neurons::add
 * (Neurons.cpp:29-48).  The neuron is appended before the duplicate check,
 * as in the reference, so a duplicate makes later simulation creation fail. */
int nemo_oracle_add_neurons(nemo_oracle_network* net, unsigned type, size_t n,
		const unsigned* idx, unsigned nargs, const float* args)
{
	if(type >= net->ntypes) return fail(NEMO_INVALID_INPUT, "Invalid neuron type id %u", type);
	neuron_coll* c = &net->types[type];
	unsigned na = c->desc->nparam + c->desc->nstate;
	if(nargs != na) {
		return fail(NEMO_INVALID_INPUT,
				"Unexpected number of parameters/state variables when adding neuron. Expected %u, found %u", na, nargs);
	}
	for(size_t i = 0; i < n; ++i) {
		if(c->n == c->cap) {
			size_t ncap = c->cap ? 2 * c->cap : 256;
			c->gidx = realloc(c->gidx, ncap * sizeof(unsigned));
			c->args = realloc(c->args, ncap * (na ? na : 1) * sizeof(float));
			if(!c->gidx || !c->args) return fail(NEMO_ALLOCATION_ERROR, "allocation failed");
			c->cap = ncap;
		}
		c->gidx[c->n] = idx[i];
		if(na) memcpy(c->args + c->n * na, args + i * na, na * sizeof(float));
		uint64_t v = ((uint64_t) type << 32) | (uint64_t) c->n;
		c->n++;
		int r = hmap_insert(&net->neurons, idx[i], v, NULL);
		if(r < 0) return fail(NEMO_ALLOCATION_ERROR, "allocation failed");
		if(r == 0) {
			net->duplicate = 1;
			net->dupIdx = idx[i];
			return fail(NEMO_INVALID_INPUT, "Duplicate neuron index %u", idx[i]);
		}
	}
	return NEMO_OK;
}

int nemo_oracle_add_neuron(nemo_oracle_network* net, unsigned type, unsigned idx,
		unsigned nargs, const float* args)
{
	return nemo_oracle_add_neurons(net, type, 1, &idx, nargs, args);
}

/* NetworkImpl::addSynapse (NetworkImpl.cpp:105-130), Axon::addSynapse (Axon.cpp:9-19) */
int nemo_oracle_add_synapses(nemo_oracle_network* net, size_t n,
		const unsigned* source, const unsigned* target, const unsigned* delay,
		const float* weight, const unsigned char* plastic, uint64_t* ids)
{
	syn_store* s = &net->syn;
	for(size_t i = 0; i < n; ++i) {
		if(delay[i] < 1) {
			return fail(NEMO_INVALID_INPUT, "Invalid delay (%u) for synapse between %u and %u",
					delay[i], source[i], target[i]);
		}
		if(s->n == s->cap) {
			size_t ncap = s->cap ? 2 * s->cap : 1024;
			s->src = realloc(s->src, ncap * sizeof(unsigned));
			s->tgt = realloc(s->tgt, ncap * sizeof(unsigned));
			s->delay = realloc(s->delay, ncap * sizeof(unsigned));
			s->weight = realloc(s->weight, ncap * sizeof(float));
			s->plastic = realloc(s->plastic, ncap);
			s->sid = realloc(s->sid, ncap * sizeof(uint32_t));
			if(!s->src || !s->tgt || !s->delay || !s->weight || !s->plastic || !s->sid)
				return fail(NEMO_ALLOCATION_ERROR, "allocation failed");
			s->cap = ncap;
		}
		uint64_t* cnt;
		if(hmap_insert(&net->axons, source[i], 0, &cnt) < 0) return fail(NEMO_ALLOCATION_ERROR, "allocation failed");
		uint32_t id = (uint32_t) (*cnt)++;
		s->src[s->n] = source[i]; s->tgt[s->n] = target[i]; s->delay[s->n] = delay[i];
		s->weight[s->n] = weight[i]; s->plastic[s->n] = plastic[i] != 0; s->sid[s->n] = id;
		s->n++;
		if(delay[i] > net->maxDelay) net->maxDelay = delay[i];
		if(ids) ids[i] = ((uint64_t) source[i] << 32) | id;
	}
	return NEMO_OK;
}

int nemo_oracle_add_synapse(nemo_oracle_network* net, unsigned source, unsigned target,
		unsigned delay, float weight, unsigned char plastic, uint64_t* id)
{
	return nemo_oracle_add_synapses(net, 1, &source, &target, &delay, &weight, &plastic, id);
}

int nemo_oracle_neuron_count(nemo_oracle_network* net, unsigned* count)
{
	size_t total = 0;
	for(unsigned t = 0; t < net->ntypes; ++t) total += net->types[t].n;
	*count = (unsigned) total;
	return NEMO_OK;
}

/* --------------------------------------------------------------------- */
/* Simulation state                                                       */

typedef struct {
	const type_desc* desc;
	unsigned netType;   /* network type id; types without neurons are skipped */
	unsigned base, n;
	float* param;   /* [nparam][n] */
	float* state;   /* [history][nstate][n]; slot cycle % history is the current one */
	unsigned* rng;  /* [n][4] */
} sim_type;

typedef struct { uint32_t target; int32_t weight; } fterm;

struct nemo_oracle_simulation {
	unsigned ncount;
	sim_type types[16];
	unsigned ntypes;
	unsigned* l2g;
	unsigned* ltype;
	hmap g2l;

	unsigned* fired;
	uint64_t* recent;
	uint64_t* delays;
	int64_t* fxE;
	int64_t* fxI;
	float* curE;
	float* curI;
	float* curExt;
	unsigned* fstim;

	/* forward matrix: rows keyed by (local source, delay), ConnectivityMatrix.hpp:228-233 */
	unsigned maxDelay;
	size_t* rowStart;   /* ncount*maxDelay + 1 */
	fterm* terms;

	/* auxiliary synapse data per global source (ConnectivityMatrix.cpp:111-117) */
	int writeOnly;
	hmap aux;            /* global source -> index into auxFirst/auxCount */
	size_t* auxFirst;    /* first iteration position of each source */
	size_t* auxCount;    /* number of synapses of each source */
	size_t nsrc;
	size_t* auxIdx;      /* position of synapse in terms[], in iteration order */
	unsigned* auxDelay;
	unsigned char* auxPlastic;
	size_t nsyn;
	uint64_t* queried;
	size_t queriedCap;

	/* STDP (StdpProcess.cpp:20-46) */
	int stdp;
	int32_t* fnPre; unsigned npre;
	int32_t* fnPost; unsigned npost;
	uint64_t potBits, depBits, prePostBits, postPreBits, postFireMask;
	int32_t minE, maxE, minI, maxI;

	/* reverse matrix of all synapses, per target, for a type that reads
	 * its sources (construction/RCM.cpp:58-99, 150-172 with STDP off):
	 * source, delay, the weight as given */
	size_t* allStart;   /* ncount + 1 */
	uint32_t* allSource;
	uint32_t* allDelay;
	float* allWeight;

	/* reverse matrix (plastic synapses only when STDP is on), per target */
	size_t* rcmStart;   /* ncount + 1 */
	uint32_t* rcmSource;
	uint32_t* rcmDelay;
	size_t* rcmForward; /* index into terms[] */
	int32_t* rcmAcc;

	unsigned long cycle;
	unsigned long timer;
	unsigned* firedList;
	size_t firedLen;
};

static unsigned local_idx(const nemo_oracle_simulation* s, unsigned g, int* ok)
{
	uint64_t* v = hmap_find(&s->g2l, g);
	if(!v) { *ok = 0; return 0; }
	*ok = 1;
	return (unsigned) *v;
}

void nemo_oracle_delete_simulation(nemo_oracle_simulation* s)
{
	if(!s) return;
	for(unsigned t = 0; t < s->ntypes; ++t) {
		free(s->types[t].param); free(s->types[t].state); free(s->types[t].rng);
	}
	free(s->l2g); free(s->ltype); hmap_free(&s->g2l);
	free(s->fired); free(s->recent); free(s->delays); free(s->fxE); free(s->fxI);
	free(s->curE); free(s->curI); free(s->curExt); free(s->fstim);
	free(s->rowStart); free(s->terms);
	hmap_free(&s->aux); free(s->auxFirst); free(s->auxCount); free(s->auxIdx); free(s->auxDelay); free(s->auxPlastic); free(s->queried);
	free(s->fnPre); free(s->fnPost);
	free(s->rcmStart); free(s->rcmSource); free(s->rcmDelay); free(s->rcmForward); free(s->rcmAcc);
	free(s->allStart); free(s->allSource); free(s->allDelay); free(s->allWeight);
	free(s->firedList);
	free(s);
}

/* Sort synapse positions by global source id, stable: this is the
 * std::map<nidx_t, Axon> iteration order of NetworkImpl::synapse_begin
 * (NetworkImpl.cpp:310-324, NetworkImpl.hpp:134). */
static size_t* iteration_order(const nemo_oracle_network* net)
{
	const syn_store* sy = &net->syn;
	size_t n = sy->n;
	size_t* order = malloc((n ? n : 1) * sizeof(size_t));
	if(!order) return NULL;
	/* two-pass LSD radix sort on the 32-bit source, 16 bits per pass */
	size_t* tmp = malloc((n ? n : 1) * sizeof(size_t));
	size_t* cnt = malloc(65537 * sizeof(size_t));
	if(!tmp || !cnt) { free(order); free(tmp); free(cnt); return NULL; }
	for(size_t i = 0; i < n; ++i) order[i] = i;
	for(int pass = 0; pass < 2; ++pass) {
		unsigned sh = 16 * pass;
		memset(cnt, 0, 65537 * sizeof(size_t));
		for(size_t i = 0; i < n; ++i) cnt[((sy->src[order[i]] >> sh) & 0xffff) + 1]++;
		for(size_t k = 0; k < 65536; ++k) cnt[k+1] += cnt[k];
		for(size_t i = 0; i < n; ++i) tmp[cnt[(sy->src[order[i]] >> sh) & 0xffff]++] = order[i];
		size_t* x = order; order = tmp; tmp = x;
	}
	free(tmp); free(cnt);
	return order;
}

static void init_kuramoto(sim_type* t);

nemo_oracle_simulation* nemo_oracle_new_simulation(nemo_oracle_network* net, nemo_oracle_configuration* conf)
{
	unsigned ncount;
	nemo_oracle_neuron_count(net, &ncount);
	/* nemo.cpp:112-118 */
	if(ncount == 0) { fail(NEMO_INVALID_INPUT, "Cannot create simulation from empty network"); return NULL; }
	if(conf->stdp && net->maxDelay + conf->npost > MAX_HISTORY) {
		/* StdpFunction.cpp:51-60 */
		fail(NEMO_INVALID_INPUT, "Max delay + postfire part of STDP function must be <= 64");
		return NULL;
	}
	/* cpu/Simulation.cpp:52-56 */
	if(net->maxDelay > 64) {
		fail(NEMO_INVALID_INPUT, "The network has synapses with delay %ums. The CPU backend supports a maximum of 64 ms", net->maxDelay);
		return NULL;
	}
	if(net->duplicate) { fail(NEMO_INVALID_INPUT, "Duplicate neuron index %u", net->dupIdx); return NULL; }

	nemo_oracle_simulation* s = calloc(1, sizeof *s);
	if(!s) { fail(NEMO_ALLOCATION_ERROR, "allocation failed"); return NULL; }
	s->ncount = ncount;
	size_t N = ncount;
	s->l2g = malloc(N * sizeof(unsigned));
	s->ltype = malloc(N * sizeof(unsigned));
	s->fired = calloc(N, sizeof(unsigned));
	s->recent = calloc(N, sizeof(uint64_t));
	s->delays = calloc(N, sizeof(uint64_t));
	s->fxE = calloc(N, sizeof(int64_t));
	s->fxI = calloc(N, sizeof(int64_t));
	s->curE = calloc(N, sizeof(float));
	s->curI = calloc(N, sizeof(float));
	s->curExt = calloc(N, sizeof(float));
	s->fstim = calloc(N, sizeof(unsigned));
	s->firedList = malloc(N * sizeof(unsigned));
	if(!s->l2g || !s->ltype || !s->fired || !s->recent || !s->delays || !s->fxE || !s->fxI
			|| !s->curE || !s->curI || !s->curExt || !s->fstim || !s->firedList) {
		nemo_oracle_delete_simulation(s);
		fail(NEMO_ALLOCATION_ERROR, "allocation failed");
		return NULL;
	}

	/* Contiguous local indices, type order then insertion order
	 * (cpu/Simulation.cpp:58-73, cpu/Neurons.cpp:26-39) */
	unsigned l = 0;
	for(unsigned t = 0; t < net->ntypes; ++t) {
		const neuron_coll* c = &net->types[t];
		if(c->n == 0) continue;
		sim_type* st = &s->types[s->ntypes++];
		st->desc = c->desc;
		st->netType = t;
		st->base = l;
		st->n = (unsigned) c->n;
		unsigned np = c->desc->nparam, ns = c->desc->nstate, na = np + ns;
		st->param = malloc((np * c->n + 1) * sizeof(float));
		st->state = calloc(c->desc->history * ns * c->n + 1, sizeof(float));
		st->rng = malloc(4 * c->n * sizeof(unsigned));
		for(size_t i = 0; i < c->n; ++i) {
			for(unsigned p = 0; p < np; ++p) st->param[p * c->n + i] = c->args[i * na + p];
			for(unsigned v = 0; v < ns; ++v) st->state[v * c->n + i] = c->args[i * na + np + v];
			s->l2g[l + i] = c->gidx[i];
			s->ltype[l + i] = s->ntypes - 1;
			hmap_insert(&s->g2l, c->gidx[i], l + i, NULL);
		}
		/* RNG seeding by local index (cpu/Neurons.cpp:41, RNG.cpp:38-63) */
		nemo_oracle_seed_states(st->base, st->n, st->rng);
		if(c->desc->kind == KIND_KURAMOTO) init_kuramoto(st);
		l += st->n;
	}

	/* Connectivity (ConnectivityMatrix.cpp:65-162) */
	const syn_store* sy = &net->syn;
	size_t S = sy->n;
	s->nsyn = S;
	s->maxDelay = net->maxDelay;
	s->writeOnly = conf->writeOnly;
	size_t* order = iteration_order(net);
	if(!order) { nemo_oracle_delete_simulation(s); fail(NEMO_ALLOCATION_ERROR, "allocation failed"); return NULL; }

	/* map endpoints; every source and target must exist
	 * (ConnectivityMatrix.cpp:83-86 + verifySynapseTerminals :166-189) */
	unsigned* lsrc = malloc((S ? S : 1) * sizeof(unsigned));
	unsigned* ltgt = malloc((S ? S : 1) * sizeof(unsigned));
	int32_t* fxw = malloc((S ? S : 1) * sizeof(int32_t));
	for(size_t k = 0; k < S; ++k) {
		size_t i = order[k];
		int ok;
		lsrc[k] = local_idx(s, sy->src[i], &ok);
		if(!ok) { fail(NEMO_INVALID_INPUT, "Non-existing neuron index %u", sy->src[i]); goto bad; }
		ltgt[k] = local_idx(s, sy->tgt[i], &ok);
		if(!ok) { fail(NEMO_INVALID_INPUT, "Non-existing neuron index %u", sy->tgt[i]); goto bad; }
		if(fx_toFix(sy->weight[i], &fxw[k]) != NEMO_OK) goto bad;
	}

	/* a type that reads its sources needs the reverse matrix of all synapses,
	 * which cannot coexist with STDP's (construction/RCM.cpp:90-98) */
	int needAll = 0;
	for(unsigned t = 0; t < s->ntypes; ++t) needAll |= s->types[t].desc->rcm;
	if(needAll && conf->stdp) {
		fail(NEMO_API_UNSUPPORTED, "The current version does not support a mix of STDP with neuron types which require reverse connectivity for other purposes");
		goto bad;
	}
	if(needAll) {
		s->allStart = calloc(N + 1, sizeof(size_t));
		for(size_t k = 0; k < S; ++k) s->allStart[ltgt[k] + 1]++;
		for(size_t n = 0; n < N; ++n) s->allStart[n+1] += s->allStart[n];
		s->allSource = malloc((S ? S : 1) * sizeof(uint32_t));
		s->allDelay = malloc((S ? S : 1) * sizeof(uint32_t));
		s->allWeight = malloc((S ? S : 1) * sizeof(float));
		size_t* afill = malloc((N ? N : 1) * sizeof(size_t));
		memcpy(afill, s->allStart, N * sizeof(size_t));
		for(size_t k = 0; k < S; ++k) {
			size_t p = afill[ltgt[k]]++;
			s->allSource[p] = lsrc[k];
			s->allDelay[p] = sy->delay[order[k]];
			s->allWeight[p] = sy->weight[order[k]];
		}
		free(afill);
	}

	{
		unsigned D = s->maxDelay;
		size_t nrows = N * (size_t) D;
		s->rowStart = calloc(nrows + 1, sizeof(size_t));
		s->terms = malloc((S ? S : 1) * sizeof(fterm));
		size_t* fill = malloc((nrows ? nrows : 1) * sizeof(size_t));
		size_t* pos = malloc((S ? S : 1) * sizeof(size_t));
		for(size_t k = 0; k < S; ++k) s->rowStart[(size_t) lsrc[k] * D + sy->delay[order[k]] - 1 + 1]++;
		for(size_t r = 0; r < nrows; ++r) s->rowStart[r+1] += s->rowStart[r];
		if(nrows) memcpy(fill, s->rowStart, nrows * sizeof(size_t));
		for(size_t k = 0; k < S; ++k) {
			size_t r = (size_t) lsrc[k] * D + sy->delay[order[k]] - 1;
			size_t p = fill[r]++;
			s->terms[p].target = ltgt[k];
			s->terms[p].weight = fxw[k];
			pos[k] = p;
			s->delays[lsrc[k]] |= (uint64_t) 1 << (sy->delay[order[k]] - 1); /* OutgoingDelays.cpp:70-80 */
		}
		free(fill);

		/* auxiliary per-source synapse table for queries, indexed by the
		 * per-source synapse id (ConnectivityMatrix.cpp:111-117) */
		s->auxIdx = malloc((S ? S : 1) * sizeof(size_t));
		s->auxDelay = malloc((S ? S : 1) * sizeof(unsigned));
		s->auxPlastic = malloc((S ? S : 1));
		s->auxFirst = malloc((S ? S : 1) * sizeof(size_t));
		s->auxCount = malloc((S ? S : 1) * sizeof(size_t));
		for(size_t k = 0; k < S; ++k) {
			size_t i = order[k];
			uint64_t* slot;
			if(hmap_insert(&s->aux, sy->src[i], s->nsrc, &slot) == 1) {
				s->auxFirst[s->nsrc] = k;
				s->auxCount[s->nsrc] = 0;
				s->nsrc++;
			}
			s->auxCount[*slot]++;
			s->auxIdx[k] = pos[k];
			s->auxDelay[k] = sy->delay[i];
			s->auxPlastic[k] = sy->plastic[i];
		}

		/* STDP process (StdpProcess.cpp:20-46) */
		if(conf->stdp) {
			s->stdp = 1;
			s->npre = (unsigned) conf->npre;
			s->npost = (unsigned) conf->npost;
			s->fnPre = malloc((s->npre ? s->npre : 1) * sizeof(int32_t));
			s->fnPost = malloc((s->npost ? s->npost : 1) * sizeof(int32_t));
			for(unsigned i = 0; i < s->npre; ++i) if(fx_toFix(conf->pre[i], &s->fnPre[i])) goto bad2;
			for(unsigned i = 0; i < s->npost; ++i) if(fx_toFix(conf->post[i], &s->fnPost[i])) goto bad2;
			if(fx_toFix(conf->minE, &s->minE) || fx_toFix(conf->maxE, &s->maxE)
					|| fx_toFix(conf->minI, &s->minI) || fx_toFix(conf->maxI, &s->maxI)) goto bad2;
			/* StdpFunction::getBits (StdpFunction.cpp:72-90): postfire reversed, then prefire */
			uint64_t pot = 0, dep = 0;
			unsigned b = 0;
			for(unsigned i = s->npost; i-- > 0; ++b) {
				if(conf->post[i] > 0.0f) pot |= (uint64_t) 1 << b;
				if(conf->post[i] < 0.0f) dep |= (uint64_t) 1 << b;
			}
			for(unsigned i = 0; i < s->npre; ++i, ++b) {
				if(conf->pre[i] > 0.0f) pot |= (uint64_t) 1 << b;
				if(conf->pre[i] < 0.0f) dep |= (uint64_t) 1 << b;
			}
			s->potBits = pot;
			s->depBits = dep;
			s->prePostBits = shl64(~shl64(~(uint64_t) 0, s->npre), s->npost);
			s->postPreBits = ~shl64(~(uint64_t) 0, s->npost);
			s->postFireMask = shl64(1, s->npost);

			/* reverse matrix of plastic synapses, per target in iteration
			 * order (construction/RCM.cpp:150-172) */
			s->rcmStart = calloc(N + 1, sizeof(size_t));
			size_t P = 0;
			for(size_t k = 0; k < S; ++k) if(sy->plastic[order[k]]) { s->rcmStart[ltgt[k] + 1]++; P++; }
			for(size_t n = 0; n < N; ++n) s->rcmStart[n+1] += s->rcmStart[n];
			s->rcmSource = malloc((P ? P : 1) * sizeof(uint32_t));
			s->rcmDelay = malloc((P ? P : 1) * sizeof(uint32_t));
			s->rcmForward = malloc((P ? P : 1) * sizeof(size_t));
			s->rcmAcc = calloc(P ? P : 1, sizeof(int32_t));
			size_t* rfill = malloc((N ? N : 1) * sizeof(size_t));
			memcpy(rfill, s->rcmStart, N * sizeof(size_t));
			for(size_t k = 0; k < S; ++k) {
				if(!sy->plastic[order[k]]) continue;
				size_t p = rfill[ltgt[k]]++;
				s->rcmSource[p] = lsrc[k];
				s->rcmDelay[p] = sy->delay[order[k]];
				s->rcmForward[p] = pos[k];
			}
			free(rfill);
		}
		free(pos);
	}
	free(order); free(lsrc); free(ltgt); free(fxw);
	return s;

bad2:
	free(order); free(lsrc); free(ltgt); free(fxw);
	nemo_oracle_delete_simulation(s);
	return NULL;
bad:
	free(order); free(lsrc); free(ltgt); free(fxw);
	nemo_oracle_delete_simulation(s);
	return NULL;
}

/* --------------------------------------------------------------------- */
/* Neuron plugins                                                         */

/* cpu/plugins/Izhikevich.cpp:14-95.  Parameters a,b,c,d,sigma
 * (plugins/Izhikevich.h:6-10), state u,v (:12-13). */
static void update_izhikevich(nemo_oracle_simulation* s, sim_type* t)
{
	const unsigned n = t->n, start = t->base;
	const float* a = t->param + 0 * n;
	const float* b = t->param + 1 * n;
	const float* c = t->param + 2 * n;
	const float* d = t->param + 3 * n;
	const float* sigma = t->param + 4 * n;
	float* U = t->state + 0 * n;
	float* V = t->state + 1 * n;
	int nn = (int) n;
#pragma omp parallel for default(shared)
	for(int nl = 0; nl < nn; nl++) {
		unsigned ng = start + nl;
		float I = s->curE[ng] + s->curI[ng] + s->curExt[ng];
		s->curExt[ng] = 0.0f;
		if(sigma[nl] != 0.0f) {
			I += sigma[nl] * nemo_oracle_nrand(&t->rng[4 * nl]);
		}
		s->fired[ng] = 0;
		float u = U[nl];
		float v = V[nl];
		for(unsigned k = 0; k < 4; ++k) {
			if(!s->fired[ng]) {
				/* v in double (0.04, 5.0, 140.0 are double literals), u in float */
				v += 0.25f * ((0.04 * v + 5.0) * v + 140.0 - u + I);
				u += 0.25f * (a[nl] * (b[nl] * v - u));
				s->fired[ng] = v >= 30.0;
			}
		}
		s->fired[ng] |= s->fstim[ng];
		s->fstim[ng] = 0;
		s->recent[ng] = (s->recent[ng] << 1) | (uint64_t) s->fired[ng];
		if(s->fired[ng]) {
			v = c[nl];
			u += d[nl];
		}
		U[nl] = u;
		V[nl] = v;
	}
}

/* cpu/plugins/IF_curr_exp.cpp:27-122 with the header parameter indices
 * (plugins/IF_curr_exp.h:4-20). */
static void update_if_curr_exp(nemo_oracle_simulation* s, sim_type* t)
{
	const unsigned n = t->n, start = t->base;
	const float* v_rest = t->param + 0 * n;
	const float* v_reset = t->param + 1 * n;
	const float* c_m = t->param + 2 * n;
	const float* tau_m = t->param + 3 * n;
	const float* tau_refrac = t->param + 4 * n;
	const float* tau_syn_E = t->param + 5 * n;
	const float* tau_syn_I = t->param + 6 * n;
	const float* v_thresh = t->param + 7 * n;
	const float* i_offset = t->param + 8 * n;
	float* V = t->state + 0 * n;
	float* IE = t->state + 1 * n;
	float* II = t->state + 2 * n;
	float* LF = t->state + 3 * n;
	int nn = (int) n;
#pragma omp parallel for default(shared)
	for(int nl = 0; nl < nn; nl++) {
		unsigned ng = start + nl;
		float Ie = ((1.0f - 1.0f / tau_syn_E[nl]) * IE[nl]) + s->curE[ng];
		float Ii = ((1.0f - 1.0f / tau_syn_I[nl]) * II[nl]) + s->curI[ng];
		float I = Ie + Ii + s->curExt[ng] + i_offset[nl];
		IE[nl] = Ie;
		II[nl] = Ii;
		s->curExt[ng] = 0.0f;
		float v = V[nl];
		int refractory = LF[nl] <= tau_refrac[nl];
		if(!refractory) {
			v += I / c_m[nl] + (v_rest[nl] - v) / tau_m[nl];
		}
		s->fired[ng] = (!refractory && v > v_thresh[nl]) || s->fstim[ng];
		s->fstim[ng] = 0;
		s->recent[ng] = (s->recent[ng] << 1) | (uint64_t) s->fired[ng];
		if(s->fired[ng]) {
			LF[nl] = 1;
			V[nl] = v_reset[nl];
		} else {
			LF[nl] += 1;
			V[nl] = v;
		}
	}
}

/* cpu/plugins/PoissonSource.cpp:6-30 (serial, as in the reference) */
static void update_poisson(nemo_oracle_simulation* s, sim_type* t)
{
	const float* rate = t->param;
	for(unsigned ng = t->base, nl = 0; ng < t->base + t->n; ng++, nl++) {
		unsigned p0 = (unsigned) (int64_t) (rate[nl] * (float) (1 << 16));
		unsigned p1 = nemo_oracle_urand(&t->rng[4 * nl]) & 0xffff;
		s->fired[ng] = p1 < p0 || s->fstim[ng];
		s->fstim[ng] = 0;
		s->recent[ng] = (s->recent[ng] << 1) | (uint64_t) s->fired[ng];
	}
}

/* cpu/plugins/Input.cpp:6-26 */
static void update_input(nemo_oracle_simulation* s, sim_type* t)
{
	for(unsigned n = t->base; n < t->base + t->n; n++) {
		s->fired[n] = s->fstim[n];
		s->fstim[n] = 0;
		s->recent[n] = (s->recent[n] << 1) | (uint64_t) s->fired[n];
	}
}

/* --------------------------------------------------------------------- */
/* Step: cpu/Simulation.cpp:94-111                                        */

/* deliverSpikes / deliverSpikesOne, cpu/Simulation.cpp:259-307 */
static void deliver_spikes(nemo_oracle_simulation* s)
{
	const unsigned D = s->maxDelay;
	uint64_t valid = ~shl64(~(uint64_t) 0, D);
	for(size_t src = 0; src < s->ncount; ++src) {
		uint64_t f = s->recent[src] & valid & s->delays[src];
		unsigned delay = 0;
		while(f) {
			unsigned shift = 1 + (unsigned) __builtin_ctzll(f);
			delay += shift;
			f = shr64(f, shift);
			size_t r = src * D + delay - 1;
			for(size_t k = s->rowStart[r]; k < s->rowStart[r+1]; ++k) {
				const fterm* term = &s->terms[k];
				if(term->weight >= 0) s->fxE[term->target] += term->weight;
				else s->fxI[term->target] += term->weight;
			}
		}
	}
	int nc = (int) s->ncount;
#pragma omp parallel for default(shared)
	for(int n = 0; n < nc; n++) {
		s->curE[n] = wfx_toFloat(s->fxE[n]);
		s->fxE[n] = 0;
		s->curI[n] = wfx_toFloat(s->fxI[n]);
		s->fxI[n] = 0;
	}
}

/* StdpProcess.cpp:68-124 */
static int32_t update_region(const nemo_oracle_simulation* s, uint64_t arrivals)
{
	int32_t w = 0;
	if(arrivals) {
		const unsigned NONE = ~0u;
		uint64_t vpre = arrivals & s->prePostBits;
		unsigned dt_pre = vpre ? (unsigned) __builtin_ctzll(shr64(vpre, s->npost)) : NONE;
		uint64_t vpost = arrivals & s->postPreBits;
		unsigned dt_post = vpost ? (unsigned) __builtin_clzll(shl64(vpost, 64 - s->npost)) : NONE;
		if(dt_pre < dt_post) w = s->fnPre[dt_pre];
		else if(dt_post < dt_pre) w = s->fnPost[dt_post];
	}
	return w;
}

static inline int32_t weight_change(const nemo_oracle_simulation* s, uint64_t pre)
{
	return wrap_add32(update_region(s, pre & s->potBits), update_region(s, pre & s->depBits));
}

/* IzhikevichRS has no CPU plugin in the reference (IzhikevichRS.ini:
 * backends cpu=false): this restates its CUDA plugin,
 * cuda/plugins/IzhikevichRS.cu:76-116 -- the Izhikevich update in float with
 * a = 0.02, b = 0.2, c = -65, d = 8 built in and no input noise, in source
 * order with no contraction (the reference's own build may contract).  State
 * u, v. */
static void update_izhikevich_rs(nemo_oracle_simulation* s, sim_type* t)
{
	const unsigned n = t->n, start = t->base;
	float* U = t->state + 0 * n;
	float* V = t->state + 1 * n;
	const float a = 0.02f, b = 0.2f;
	int nn = (int) n;
#pragma omp parallel for default(shared)
	for(int nl = 0; nl < nn; nl++) {
		unsigned ng = start + nl;
		float I = s->curE[ng] + s->curI[ng] + s->curExt[ng];
		s->curExt[ng] = 0.0f;
		float u = U[nl];
		float v = V[nl];
		int fired = 0;
		for(unsigned k = 0; k < 4; ++k) {
			if(!fired) {
				v += 0.25f * ((0.04f * v + 5.0f) * v + 140.0f - u + I);
				u += 0.25f * (a * (b * v - u));
				fired = v >= 30.0f;
			}
		}
		s->fired[ng] = fired || s->fstim[ng];
		s->fstim[ng] = 0;
		s->recent[ng] = (s->recent[ng] << 1) | (uint64_t) s->fired[ng];
		if(s->fired[ng]) {
			v = -65.0f;
			u += 8.0f;
		}
		U[nl] = u;
		V[nl] = v;
	}
}

/* Kuramoto oscillators, cpu/plugins/Kuramoto.cpp (plugins/Kuramoto.h):
 * parameter the frequency, state the phase, kept for the last 32 cycles.
 * Each update integrates the phase with one fourth-order Runge-Kutta step
 * whose coupling sums, over the incoming synapses in reverse-matrix order,
 * weight x sinf(source phase at emission - target phase); the source phase
 * is the one at cycle - (delay - 1).  The neuron never fires. */
#define KURAMOTO_HISTORY 32

static float* kuramoto_phase(sim_type* t, unsigned long cycle)
{
	return t->state + (size_t) (cycle % KURAMOTO_HISTORY) * t->n;
}

/* sumN (cpu/plugins/Kuramoto.cpp:17-30) */
static float kuramoto_coupling(nemo_oracle_simulation* s, sim_type* t, unsigned ng, float targetPhase)
{
	float sum = 0.0f;
	for(size_t k = s->allStart[ng]; k < s->allStart[ng + 1]; ++k) {
		const float* src = kuramoto_phase(t, s->cycle - (s->allDelay[k] - 1));
		sum += s->allWeight[k] * sinf(src[s->allSource[k] - t->base] - targetPhase);
	}
	return sum;
}

/* cpu_update_neurons (cpu/plugins/Kuramoto.cpp:78-124) */
static void update_kuramoto(nemo_oracle_simulation* s, sim_type* t)
{
	const float* frequency = t->param;
	const float* phase0 = kuramoto_phase(t, s->cycle);
	float* phase1 = kuramoto_phase(t, s->cycle + 1);
	for(unsigned nl = 0; nl < t->n; ++nl) {
		const unsigned ng = t->base + nl;
		const float f = frequency[nl];
		float targetPhase = phase0[nl];
		float k0 = f + kuramoto_coupling(s, t, ng, targetPhase);
		float k1 = f + kuramoto_coupling(s, t, ng, targetPhase + k0 * 0.5f);
		float k2 = f + kuramoto_coupling(s, t, ng, targetPhase + k1 * 0.5f);
		float k3 = f + kuramoto_coupling(s, t, ng, targetPhase + k2);
		targetPhase += (k0 + 2 * k1 + 2 * k2 + k3) / 6.0f;
		phase1[nl] = fmodf(targetPhase, 2.0f * M_PI) + (targetPhase < 0.0f ? 2.0f * M_PI : 0.0f);
	}
}

/* cpu_init_neurons (cpu/plugins/Kuramoto.cpp:131-151): the history before
 * cycle 0, run backwards without coupling */
static void init_kuramoto(sim_type* t)
{
	const float* frequency = t->param;
	for(unsigned k = 0; k < KURAMOTO_HISTORY - 1; k++) {
		const unsigned current = 0U - k, previous = 0U - (k + 1U);
		const float* phase0 = t->state + (size_t) (current % KURAMOTO_HISTORY) * t->n;
		float* phase1 = t->state + (size_t) (previous % KURAMOTO_HISTORY) * t->n;
		for(unsigned nl = 0; nl < t->n; nl++) {
			float phase = phase0[nl] - frequency[nl];
			phase1[nl] = fmodf(phase, 2.0f * M_PI) + (phase < 0.0f ? 2.0f * M_PI : 0.0f);
		}
	}
}

/* ConnectivityMatrix::accumulateStdp, ConnectivityMatrix.cpp:193-227 */
static void accumulate_stdp(nemo_oracle_simulation* s)
{
	if(!s->stdp) return;
	for(size_t tgt = 0; tgt < s->ncount; ++tgt) {
		if(!(s->recent[tgt] & s->postFireMask)) continue;
		for(size_t k = s->rcmStart[tgt]; k < s->rcmStart[tgt+1]; ++k) {
			uint64_t pre = shr64(s->recent[s->rcmSource[k]], s->rcmDelay[k]);
			int32_t dw = weight_change(s, pre);
			if(dw != 0) s->rcmAcc[k] = wrap_add32(s->rcmAcc[k], dw);
		}
	}
}

static void fire(nemo_oracle_simulation* s)
{
	deliver_spikes(s);
	for(unsigned t = 0; t < s->ntypes; ++t) {
		sim_type* st = &s->types[t];
		switch(st->desc->kind) {
			case KIND_IZHIKEVICH: update_izhikevich(s, st); break;
			case KIND_IF_CURR_EXP: update_if_curr_exp(s, st); break;
			case KIND_POISSON: update_poisson(s, st); break;
			case KIND_INPUT: update_input(s, st); break;
			case KIND_IZHIKEVICH_RS: update_izhikevich_rs(s, st); break;
			case KIND_KURAMOTO: update_kuramoto(s, st); break;
		}
	}
	accumulate_stdp(s);
	/* setFiring, cpu/Simulation.cpp:200-208 */
	s->firedLen = 0;
	for(unsigned n = 0; n < s->ncount; ++n) {
		if(s->fired[n]) s->firedList[s->firedLen++] = s->l2g[n];
	}
	s->cycle++;
	s->timer++;
}

/* nemo_c.cpp:440-461: firing stimulus, then current stimulus, then fire */
int nemo_oracle_step(nemo_oracle_simulation* s,
		const unsigned* fstim, size_t nf,
		const unsigned* inidx, const float* icur, size_t ni,
		const unsigned** fired, size_t* nfired)
{
	int ok;
	for(size_t i = 0; i < nf; ++i) {
		unsigned l = local_idx(s, fstim[i], &ok);
		if(!ok) return fail(NEMO_INVALID_INPUT, "Non-existing neuron index %u", fstim[i]);
		s->fstim[l] = 1;
	}
	for(size_t i = 0; i < ni; ++i) {
		unsigned l = local_idx(s, inidx[i], &ok);
		if(!ok) return fail(NEMO_INVALID_INPUT, "Non-existing neuron index %u", inidx[i]);
		s->curExt[l] = icur[i];
	}
	fire(s);
	if(fired) *fired = s->firedLen ? s->firedList : NULL;
	if(nfired) *nfired = s->firedLen;
	return NEMO_OK;
}

int nemo_oracle_run(nemo_oracle_simulation* s, unsigned steps, unsigned stdp_period, float reward,
		unsigned* counts, unsigned* ids, size_t cap, size_t* len)
{
	size_t total = 0;
	for(unsigned t = 0; t < steps; ++t) {
		fire(s);
		if(counts) counts[t] = (unsigned) s->firedLen;
		if(ids) {
			if(total + s->firedLen > cap) return fail(NEMO_BUFFER_OVERFLOW, "fired id buffer too small");
			memcpy(ids + total, s->firedList, s->firedLen * sizeof(unsigned));
		}
		total += s->firedLen;
		if(stdp_period && (t + 1) % stdp_period == 0) {
			int r = nemo_oracle_apply_stdp(s, reward);
			if(r) return r;
		}
	}
	if(len) *len = total;
	return NEMO_OK;
}

/* StdpProcess::updatedWeight, StdpProcess.cpp:128-138 */
static inline int32_t updated_weight(const nemo_oracle_simulation* s, int32_t w, int32_t dw)
{
	int32_t nw = 0;
	int32_t sum = wrap_add32(w, dw);
	if(w > 0) {
		int32_t x = sum > s->minE ? sum : s->minE;
		nw = s->maxE < x ? s->maxE : x;
	} else if(w < 0) {
		int32_t x = sum > s->maxI ? sum : s->maxI;
		nw = s->minI < x ? s->minI : x;
	}
	return nw;
}

/* ConnectivityMatrix::applyStdp, ConnectivityMatrix.cpp:241-294 */
int nemo_oracle_apply_stdp(nemo_oracle_simulation* s, float reward)
{
	if(!s->stdp) return fail(NEMO_LOGIC_ERROR, "applyStdp called, but no STDP model specified");
	int32_t R;
	int r = fx_toFix(reward, &R);
	if(r) return r;
	if(R == 0 && reward != 0) {
		return fail(NEMO_INVALID_INPUT, "STDP reward rounded down to zero. The smallest valid reward is %f",
				(double) fx_toFloat(1));
	}
	size_t P = s->rcmStart[s->ncount];
	if(R == 0) memset(s->rcmAcc, 0, P * sizeof(int32_t));
	for(size_t k = 0; k < P; ++k) {
		int32_t* w = &s->terms[s->rcmForward[k]].weight;
		int32_t nw = updated_weight(s, *w, fx_mul(R, s->rcmAcc[k]));
		if(*w != nw) *w = nw;
		s->rcmAcc[k] = 0;
	}
	return NEMO_OK;
}

/* --------------------------------------------------------------------- */
/* Queries                                                                */

static int locate(nemo_oracle_simulation* s, unsigned g, sim_type** t, unsigned* i)
{
	int ok;
	unsigned l = local_idx(s, g, &ok);
	if(!ok) return fail(NEMO_INVALID_INPUT, "Non-existing neuron index %u", g);
	*t = &s->types[s->ltype[l]];
	*i = l - (*t)->base;
	return NEMO_OK;
}

/* the state of the current cycle (cpu/Neurons.cpp:80-92, :123) */
static float* current_state(nemo_oracle_simulation* s, sim_type* t)
{
	return t->state + (size_t) (s->cycle % t->desc->history) * t->desc->nstate * t->n;
}

int nemo_oracle_get_neuron_state(nemo_oracle_simulation* s, unsigned g, unsigned var, float* val)
{
	sim_type* t; unsigned i;
	int r = locate(s, g, &t, &i); if(r) return r;
	if(var >= t->desc->nstate) return fail(NEMO_INVALID_INPUT, "Invalid state variable index %u", var);
	*val = current_state(s, t)[var * t->n + i];
	return NEMO_OK;
}

int nemo_oracle_get_neuron_parameter(nemo_oracle_simulation* s, unsigned g, unsigned p, float* val)
{
	sim_type* t; unsigned i;
	int r = locate(s, g, &t, &i); if(r) return r;
	if(p >= t->desc->nparam) return fail(NEMO_INVALID_INPUT, "Invalid parameter index %u", p);
	*val = t->param[p * t->n + i];
	return NEMO_OK;
}

int nemo_oracle_get_membrane_potential(nemo_oracle_simulation* s, unsigned g, float* val)
{
	sim_type* t; unsigned i;
	int r = locate(s, g, &t, &i); if(r) return r;
	return nemo_oracle_get_neuron_state(s, g, t->desc->mpot, val);
}

int nemo_oracle_set_neuron_state(nemo_oracle_simulation* s, unsigned g, unsigned var, float val)
{
	sim_type* t; unsigned i;
	int r = locate(s, g, &t, &i); if(r) return r;
	if(var >= t->desc->nstate) return fail(NEMO_INVALID_INPUT, "Invalid state variable index %u", var);
	current_state(s, t)[var * t->n + i] = val;
	return NEMO_OK;
}

int nemo_oracle_set_neuron_parameter(nemo_oracle_simulation* s, unsigned g, unsigned p, float val)
{
	sim_type* t; unsigned i;
	int r = locate(s, g, &t, &i); if(r) return r;
	if(p >= t->desc->nparam) return fail(NEMO_INVALID_INPUT, "Invalid parameter index %u", p);
	t->param[p * t->n + i] = val;
	return NEMO_OK;
}

/* cpu/Neurons.cpp:52-76 */
int nemo_oracle_set_neuron(nemo_oracle_simulation* s, unsigned g, unsigned nargs, const float* args)
{
	sim_type* t; unsigned i;
	int r = locate(s, g, &t, &i); if(r) return r;
	unsigned np = t->desc->nparam, ns = t->desc->nstate;
	if(nargs != np + ns) {
		return fail(NEMO_INVALID_INPUT,
				"Unexpected number of parameters/state variables when modifying neuron. Expected %u, found %u", np + ns, nargs);
	}
	for(unsigned p = 0; p < np; ++p) t->param[p * t->n + i] = args[p];
	for(unsigned v = 0; v < ns; ++v) current_state(s, t)[v * t->n + i] = args[np + v];
	return NEMO_OK;
}

/* ConnectivityMatrix.cpp:298-331 */
int nemo_oracle_get_synapses_from(nemo_oracle_simulation* s, unsigned source, const uint64_t** ids, size_t* len)
{
	if(s->writeOnly) return fail(NEMO_INVALID_INPUT, "Cannot read synapse state if simulation configured with write-only synapses");
	uint64_t* info = hmap_find(&s->aux, source);
	size_t n = 0;
	if(!info) {
		int ok; (void) local_idx(s, source, &ok);
		if(!ok) return fail(NEMO_INVALID_INPUT, "Non-existing source neuron id (%u) in synapse id query", source);
	} else {
		n = s->auxCount[*info];
	}
	if(n > s->queriedCap) {
		free(s->queried);
		s->queried = malloc(n * sizeof(uint64_t));
		s->queriedCap = n;
	}
	for(size_t i = 0; i < n; ++i) s->queried[i] = ((uint64_t) source << 32) | i;
	*ids = n ? s->queried : NULL;
	*len = n;
	return NEMO_OK;
}

/* ConnectivityMatrix::axonTerminalAux, ConnectivityMatrix.cpp:343-360 */
static int aux_lookup(nemo_oracle_simulation* s, uint64_t id, size_t* k)
{
	if(s->writeOnly) return fail(NEMO_INVALID_INPUT, "Cannot read synapse state if simulation configured with write-only synapses");
	unsigned src = (unsigned) (id >> 32);
	uint32_t sid = (uint32_t) (id & 0xffffffffu);
	uint64_t* info = hmap_find(&s->aux, src);
	if(!info) return fail(NEMO_INVALID_INPUT, "Non-existing neuron id (%u) in synapse query", src);
	if(sid >= s->auxCount[*info]) return fail(NEMO_UNKNOWN_ERROR, "vector::_M_range_check");
	*k = s->auxFirst[*info] + sid;
	return NEMO_OK;
}

int nemo_oracle_get_synapse_target(nemo_oracle_simulation* s, uint64_t id, unsigned* target)
{
	size_t k; int r = aux_lookup(s, id, &k); if(r) return r;
	*target = s->l2g[s->terms[s->auxIdx[k]].target];
	return NEMO_OK;
}

int nemo_oracle_get_synapse_delay(nemo_oracle_simulation* s, uint64_t id, unsigned* delay)
{
	size_t k; int r = aux_lookup(s, id, &k); if(r) return r;
	*delay = s->auxDelay[k];
	return NEMO_OK;
}

int nemo_oracle_get_synapse_weight(nemo_oracle_simulation* s, uint64_t id, float* weight)
{
	size_t k; int r = aux_lookup(s, id, &k); if(r) return r;
	*weight = fx_toFloat(s->terms[s->auxIdx[k]].weight);
	return NEMO_OK;
}

int nemo_oracle_get_synapse_plastic(nemo_oracle_simulation* s, uint64_t id, unsigned char* plastic)
{
	size_t k; int r = aux_lookup(s, id, &k); if(r) return r;
	*plastic = s->auxPlastic[k];
	return NEMO_OK;
}

int nemo_oracle_get_all_weights_fx(nemo_oracle_simulation* s, int32_t* out, size_t cap, size_t* len)
{
	if(cap < s->nsyn) return fail(NEMO_BUFFER_OVERFLOW, "weight buffer too small");
	for(size_t k = 0; k < s->nsyn; ++k) out[k] = s->terms[s->auxIdx[k]].weight;
	*len = s->nsyn;
	return NEMO_OK;
}

int nemo_oracle_get_type_state(nemo_oracle_simulation* s, unsigned type, float* out, size_t cap, size_t* len)
{
	for(unsigned t = 0; t < s->ntypes; ++t) {
		if(s->types[t].netType != type) continue;
		size_t n = (size_t) s->types[t].n * s->types[t].desc->nstate;
		if(cap < n) return fail(NEMO_BUFFER_OVERFLOW, "state buffer too small");
		memcpy(out, current_state(s, &s->types[t]), n * sizeof(float));
		*len = n;
		return NEMO_OK;
	}
	*len = 0;
	return NEMO_OK;
}

int nemo_oracle_elapsed_simulation(nemo_oracle_simulation* s, unsigned long* elapsed)
{
	*elapsed = s->timer;
	return NEMO_OK;
}

int nemo_oracle_reset_timer(nemo_oracle_simulation* s)
{
	s->timer = 0;
	return NEMO_OK;
}

/* --------------------------------------------------------------------- */
/* The reference's random network generator, src/examples/random.cpp:29-88 */

/* boost::uniform_int<>(lo, hi) over a 32-bit engine (Boost >= 1.47
 * uniform_int_distribution: bucketed division with rejection; no draw at
 * all when lo == hi) */
static unsigned uniform_int_u(mt19937* g, unsigned lo, unsigned hi)
{
	uint32_t range = hi - lo;
	if(range == 0) return lo;
	if(range == 0xffffffffu) return lo + mt_next(g);
	uint32_t bucket = 0xffffffffu / (range + 1u);
	if(0xffffffffu % (range + 1u) == range) bucket++;
	for(;;) {
		uint32_t r = mt_next(g) / bucket;
		if(r <= range) return lo + r;
	}
}

/* boost::uniform_real<double>(0, 1) over a 32-bit engine: x / 2^32 */
static double uniform_01(mt19937* g) { return (double) mt_next(g) / 4294967296.0; }

/* Arguments of Network::addSynapse are evaluated right to left, as GCC does
 * on x86-64 for random.cpp:78 and :83. */
int nemo_oracle_example_random(nemo_oracle_network** out, unsigned ncount, unsigned scount,
		unsigned dmax, int stdp)
{
	return nemo_oracle_example_random_ex(out, ncount, scount, dmax, stdp, 5489u, 5.0f, 2.0f);
}

/* the same with the generator seed and the two noise sigmas as parameters */
int nemo_oracle_example_random_ex(nemo_oracle_network** out, unsigned ncount, unsigned scount,
		unsigned dmax, int stdp, unsigned seed, float sigmaExc, float sigmaInh)
{
	nemo_oracle_network* net = nemo_oracle_new_network();
	if(!net) return fail(NEMO_ALLOCATION_ERROR, "allocation failed");
	unsigned iz;
	nemo_oracle_add_neuron_type(net, "Izhikevich", &iz);
	mt19937 g;
	mt_seed(&g, seed);
	unsigned* tgt = malloc((scount ? scount : 1) * sizeof(unsigned));
	unsigned* dly = malloc((scount ? scount : 1) * sizeof(unsigned));
	unsigned* src = malloc((scount ? scount : 1) * sizeof(unsigned));
	float* w = malloc((scount ? scount : 1) * sizeof(float));
	unsigned char* pl = malloc(scount ? scount : 1);
	int r = NEMO_OK;
	for(unsigned nidx = 0; nidx < ncount && r == NEMO_OK; ++nidx) {
		float v = -65.0f;
		float args[7];
		int exc = nidx < (ncount * 4) / 5;
		if(exc) {
			/* addExcitatoryNeuron, random.cpp:29-42 */
			float a = 0.02f, b = 0.2f;
			float r1 = (float) uniform_01(&g);
			float r2 = (float) uniform_01(&g);
			float c = v + 15.0f * r1 * r1;
			float d = 8.0f - 6.0f * r2 * r2;
			float u = b * v;
			float sigma = sigmaExc;
			float x[7] = { a, b, c, d, sigma, u, v };
			memcpy(args, x, sizeof x);
		} else {
			/* addInhibitoryNeuron, random.cpp:46-59 */
			float r1 = (float) uniform_01(&g);
			float a = 0.02f + 0.08f * r1;
			float r2 = (float) uniform_01(&g);
			float b = 0.25f - 0.05f * r2;
			float c = v;
			float d = 2.0f;
			float u = b * v;
			float sigma = sigmaInh;
			float x[7] = { a, b, c, d, sigma, u, v };
			memcpy(args, x, sizeof x);
		}
		r = nemo_oracle_add_neuron(net, iz, nidx, 7, args);
		for(unsigned s = 0; s < scount; ++s) {
			src[s] = nidx;
			if(exc) {
				w[s] = 0.5f * (float) uniform_01(&g);
				dly[s] = uniform_int_u(&g, 1, dmax);
				tgt[s] = uniform_int_u(&g, 0, ncount - 1);
				pl[s] = (unsigned char) (stdp != 0);
			} else {
				w[s] = (float) (-uniform_01(&g));
				tgt[s] = uniform_int_u(&g, 0, ncount - 1);
				dly[s] = 1;
				pl[s] = 0;
			}
		}
		if(r == NEMO_OK) r = nemo_oracle_add_synapses(net, scount, src, tgt, dly, w, pl, NULL);
	}
	free(tgt); free(dly); free(src); free(w); free(pl);
	if(r != NEMO_OK) { nemo_oracle_delete_network(net); return r; }
	*out = net;
	return NEMO_OK;
}

/* Copy out the network's synapses in insertion order (for cross-checking a
 * generator against another implementation). */
int nemo_oracle_network_synapses(nemo_oracle_network* net, size_t cap,
		unsigned* source, unsigned* target, unsigned* delay, float* weight,
		unsigned char* plastic, size_t* len)
{
	const syn_store* s = &net->syn;
	*len = s->n;
	if(cap < s->n) return fail(NEMO_BUFFER_OVERFLOW, "buffer too small");
	memcpy(source, s->src, s->n * sizeof(unsigned));
	memcpy(target, s->tgt, s->n * sizeof(unsigned));
	memcpy(delay, s->delay, s->n * sizeof(unsigned));
	memcpy(weight, s->weight, s->n * sizeof(float));
	memcpy(plastic, s->plastic, s->n);
	return NEMO_OK;
}

size_t nemo_oracle_network_synapse_count(nemo_oracle_network* net) { return net->syn.n; }
