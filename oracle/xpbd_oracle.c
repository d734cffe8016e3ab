/*
 * CPU oracle for the XPBD Gaussian-graph solver step — TEST INFRASTRUCTURE ONLY.
 * See xpbd_oracle.h.  All citations are to the reference project:
 *   forward.cu  = native/solver_core/cuda_rasterizer/forward.cu
 *   capi        = native/xpbd_capi.cu
 * The arithmetic is FP32 (FP64 where the reference uses double) and keeps the
 * reference's expression order; glm's column-major conventions are mirrored by the
 * m3 type (m[col][row]).
 */
#define _GNU_SOURCE
#include "xpbd_oracle.h"

#include <float.h>
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------------- */
/* small vector / matrix helpers (forward.cu:4949-4969, glm type_mat3x3.inl)  */
/* ------------------------------------------------------------------------- */
typedef struct { float x, y, z; } f3;
typedef struct { float m[3][3]; } m3; /* glm layout: m[col][row] */

static inline f3 mk3(float x, float y, float z) { f3 r = { x, y, z }; return r; }
static inline f3 f3_add(f3 a, f3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline f3 f3_sub(f3 a, f3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline f3 f3_mul(f3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
static inline float f3_len(f3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline float f3_dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float f3_len2(f3 a) { return f3_dot(a, a); }
static inline int f3_finite(f3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
static inline float vget(f3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

static inline m3 m3_zero(void) { m3 r; memset(&r, 0, sizeof(r)); return r; }
static inline m3 m3_diag(float d) { m3 r = m3_zero(); r.m[0][0] = r.m[1][1] = r.m[2][2] = d; return r; }
/* A += outerProduct(p, q): O[c][r] = p[r] * q[c] */
static inline void m3_add_outer(m3* A, f3 p, f3 q)
{
	for (int c = 0; c < 3; ++c)
		for (int r = 0; r < 3; ++r) A->m[c][r] += vget(p, r) * vget(q, c);
}
static inline f3 m3_mulv(const m3* M, f3 v)
{
	return mk3(M->m[0][0] * v.x + M->m[1][0] * v.y + M->m[2][0] * v.z,
		M->m[0][1] * v.x + M->m[1][1] * v.y + M->m[2][1] * v.z,
		M->m[0][2] * v.x + M->m[1][2] * v.y + M->m[2][2] * v.z);
}
static inline m3 m3_mul(const m3* A, const m3* B)
{
	m3 R;
	for (int c = 0; c < 3; ++c)
		for (int r = 0; r < 3; ++r)
			R.m[c][r] = A->m[0][r] * B->m[c][0] + A->m[1][r] * B->m[c][1] + A->m[2][r] * B->m[c][2];
	return R;
}
static inline m3 m3_transpose(const m3* M)
{
	m3 T;
	for (int c = 0; c < 3; ++c)
		for (int r = 0; r < 3; ++r) T.m[c][r] = M->m[r][c];
	return T;
}
static inline m3 m3_scale(const m3* M, float s)
{
	m3 R;
	for (int c = 0; c < 3; ++c)
		for (int r = 0; r < 3; ++r) R.m[c][r] = M->m[c][r] * s;
	return R;
}
static inline m3 m3_divs(const m3* M, float s)
{
	m3 R;
	for (int c = 0; c < 3; ++c)
		for (int r = 0; r < 3; ++r) R.m[c][r] = M->m[c][r] / s;
	return R;
}
static inline m3 m3_addm(const m3* A, const m3* B)
{
	m3 R;
	for (int c = 0; c < 3; ++c)
		for (int r = 0; r < 3; ++r) R.m[c][r] = A->m[c][r] + B->m[c][r];
	return R;
}
static inline float m3_det(const m3* M)
{
	const float(*m)[3] = M->m;
	return +m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2])
		- m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2])
		+ m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
}

/* inverse3x3_safe (forward.cu:1696-1719) */
static int inverse3x3_safe(const m3* M, m3* inv, float eps_det)
{
	const float(*m)[3] = M->m;
	float a00 = m[0][0], a01 = m[0][1], a02 = m[0][2];
	float a10 = m[1][0], a11 = m[1][1], a12 = m[1][2];
	float a20 = m[2][0], a21 = m[2][1], a22 = m[2][2];
	float det = a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) + a02 * (a10 * a21 - a11 * a20);
	if (fabs(det) < eps_det) return 0;
	float invdet = 1.0f / det;
	inv->m[0][0] = (a11 * a22 - a12 * a21) * invdet;
	inv->m[0][1] = -(a01 * a22 - a02 * a21) * invdet;
	inv->m[0][2] = (a01 * a12 - a02 * a11) * invdet;
	inv->m[1][0] = -(a10 * a22 - a12 * a20) * invdet;
	inv->m[1][1] = (a00 * a22 - a02 * a20) * invdet;
	inv->m[1][2] = -(a00 * a12 - a02 * a10) * invdet;
	inv->m[2][0] = (a10 * a21 - a11 * a20) * invdet;
	inv->m[2][1] = -(a00 * a21 - a01 * a20) * invdet;
	inv->m[2][2] = (a00 * a11 - a01 * a10) * invdet;
	return 1;
}

/* jacobiEigenDecomposition3x3 (forward.cu:782-870), row-major A, cyclic-max float Jacobi */
static void jacobi_eig3(const float A_in[3][3], float ev[3], float V[3][3])
{
	float A[3][3];
	for (int i = 0; i < 3; ++i)
		for (int j = 0; j < 3; ++j) A[i][j] = A_in[i][j];
	for (int i = 0; i < 3; ++i)
		for (int j = 0; j < 3; ++j) V[i][j] = (i == j) ? 1.0f : 0.0f;
	for (int iter = 0; iter < 50; ++iter) {
		int p = 0, q = 1;
		float maxOff = fabsf(A[0][1]);
		if (fabsf(A[0][2]) > maxOff) { p = 0; q = 2; maxOff = fabsf(A[0][2]); }
		if (fabsf(A[1][2]) > maxOff) { p = 1; q = 2; maxOff = fabsf(A[1][2]); }
		if (maxOff < 1e-6f) break;
		float app = A[p][p], aqq = A[q][q], apq = A[p][q];
		float phi = 0.5f * (aqq - app) / (apq + 1e-20f);
		float t = (phi >= 0.0f) ? (1.0f / (phi + sqrtf(1.0f + phi * phi))) : (1.0f / (phi - sqrtf(1.0f + phi * phi)));
		float c = 1.0f / sqrtf(1.0f + t * t);
		float s = t * c;
		float app_new = app - t * apq;
		float aqq_new = aqq + t * apq;
		A[p][p] = app_new;
		A[q][q] = aqq_new;
		A[p][q] = A[q][p] = 0.0f;
		for (int r = 0; r < 3; ++r) {
			if (r == p || r == q) continue;
			float arp = A[r][p], arq = A[r][q];
			A[r][p] = A[p][r] = c * arp - s * arq;
			A[r][q] = A[q][r] = c * arq + s * arp;
		}
		for (int r = 0; r < 3; ++r) {
			float vrp = V[r][p], vrq = V[r][q];
			V[r][p] = c * vrp - s * vrq;
			V[r][q] = s * vrp + c * vrq;
		}
	}
	ev[0] = A[0][0]; ev[1] = A[1][1]; ev[2] = A[2][2];
	for (int i = 0; i < 2; ++i)
		for (int j = i + 1; j < 3; ++j)
			if (ev[i] > ev[j]) {
				float tmp = ev[i]; ev[i] = ev[j]; ev[j] = tmp;
				for (int r = 0; r < 3; ++r) { float t2 = V[r][i]; V[r][i] = V[r][j]; V[r][j] = t2; }
			}
}

/* eigenDecomposition_glm (forward.cu:871-901): glm in/out, eigenvectors as columns */
static void eig_glm(const m3* A, f3* evals, m3* evecs)
{
	float Ar[3][3], ev[3], V[3][3];
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c) Ar[r][c] = A->m[c][r];
	jacobi_eig3(Ar, ev, V);
	*evals = mk3(ev[0], ev[1], ev[2]);
	for (int c = 0; c < 3; ++c)
		for (int r = 0; r < 3; ++r) evecs->m[c][r] = V[r][c];
}

/* sigmaScaleAndShapeDet (forward.cu:7666-7676) */
static int sigma_scale_det(const m3* S, float* outScale, float* outDetHat)
{
	const float s = (S->m[0][0] + S->m[1][1] + S->m[2][2]) * (1.0f / 3.0f);
	if (!isfinite(s) || s <= 1e-24f) return 0;
	m3 Sh = m3_divs(S, s);
	const float detHat = m3_det(&Sh);
	if (!isfinite(detHat) || detHat <= 1e-6f) return 0;
	*outScale = s;
	*outDetHat = detHat;
	return 1;
}

/* storeSym3 / loadSym3 (forward.cu:7632-7652): [xx, yy, zz, xy, xz, yz] */
static inline void store_sym3(float* dst, const m3* S)
{
	dst[0] = S->m[0][0]; dst[1] = S->m[1][1]; dst[2] = S->m[2][2];
	dst[3] = S->m[1][0]; dst[4] = S->m[2][0]; dst[5] = S->m[2][1];
}
static inline m3 load_sym3(const float* s)
{
	m3 S = m3_zero();
	S.m[0][0] = s[0]; S.m[1][1] = s[1]; S.m[2][2] = s[2];
	S.m[0][1] = S.m[1][0] = s[3];
	S.m[0][2] = S.m[2][0] = s[4];
	S.m[1][2] = S.m[2][1] = s[5];
	return S;
}

/* warpAllSum (forward.cu:8696-8700) emulated over 32 lanes: butterfly, all lanes equal */
static float warp_allsum(const float* in)
{
	float v[32], nv[32];
	memcpy(v, in, sizeof(v));
	for (int o = 16; o > 0; o >>= 1) {
		for (int l = 0; l < 32; ++l) nv[l] = v[l] + v[l ^ o];
		memcpy(v, nv, sizeof(v));
	}
	return v[0];
}

/* ------------------------------------------------------------------------- */
/* state (capi:17-29 singleton; forward.cu:38-612, 3535-3637 file statics)    */
/* ------------------------------------------------------------------------- */
#define MAX_KIN 32
#define KIN_ACC 7
#define SC_MAX 32
typedef struct {
	float R[9], t[3], h[3];
	int type;
	float Rp[9], tp[3];
} kin_t;

static struct {
	/* created inputs */
	int n, n_edges;
	float* pos_in;
	float* scales;
	float* rots;
	float* opacity;
	int* edges;
	float* edge_rest;
	float* edge_stiff;
	int created, built, stepped;
	char err[512];
	/* graph CSR (loadGraph) */
	int m;
	int *off, *cnt, *nbr;
	float *ndist, *nstiff;
	/* state */
	f3 *pos_curr, *pos_next, *pos_tmp, *pos_rest, *vel;
	float *inv_mass, *density, *lam_a, *lam_b;
	/* volume */
	int *vol_off, *vol_cnt, *vol_idx;
	long long vol_total;
	int *rev_off, *rev_cnt, *rev_idx;
	long long rev_total;
	float *sigma_rest, *det_rest, *v_rest, *rest_len, *lam_vol;
	int* mat_type;
	f3* cl_c;
	float *cl_sinv, *cl_coef;
	int leader_count;
	float avg_members;
	int* vol_gs_order;
	int* vol_gs_color_off;
	int vol_gs_ncolors, vol_gs_clusters;
	/* distance GS */
	int gs_nedges, gs_ncolors;
	int* gs_edge; /* 2 per edge */
	float *gs_rest, *gs_stiff, *gs_lam;
	int* gs_color_off;
	/* attach (forward.cu:6759-6788) */
	int att_active;
	float* inv_mass_saved;
	/* self-collision (forward.cu:223-269) */
	float sc_spacing;
	int sc_table, sc_bits;
	unsigned int *sc_keys, *sc_keys_sorted;
	int *sc_idx_sorted, *sc_cell_start, *sc_cell_end, *sc_contact, *sc_count;
	f3 *sc_dp, *sc_dp_cross;
	float sc_reach;
	int sc_contacts, sc_overflow, sc_active;
	int* obj_id;
	int obj_k;
	/* J stats */
	float jvw_mean, jvw_std;
	/* ChainMail arrival times (forward.cu:3542; 1e9 = not reached, forward.cu:2717) */
	float *cm_time, *cm_time_next;
	/* object mode (forward.cu:164-209, 11376-11440): rest cache, fit state, boxes, weights,
	 * the frame's cross-object self-collision corrections, the self-collision active set */
	int obj_cache;
	float *obj_c0, *obj_params, *obj_disp, *obj_boxes, *obj_w;
	double *obj_q, *obj_sumq, *obj_shift;
	int* obj_count;
	int obj_shift_valid;
	f3* obj_accum;
	unsigned char* sc_act;
	/* ellipsoid contact shapes (forward.cu:150-160; xpbd_capi.cu:25-27, 181-191):
	 * M = k^2 Sigma [6 per Gaussian: xx xy xz yy yz zz], longest semi-axis, ground radius */
	int contact_on, contact_col, contact_ground, contact_n;
	float contact_tau, contact_cap;
	float *contact_M, *contact_rmax, *contact_rg;
} S;

/* press harness: the squash statics of forward.cu:530-568 in press mode; they outlive
 * create / destroy like the reference's */
static struct {
	int active, axis, from_lo, ckpt, dwell, autolog;
	float lo, hi, cur, max, ramp;
} Q = { 0, 1, 0, 0, 0, 1, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f };

/* parameters: file statics of forward.cu with their defaults (forward.cu:53-92, 224-265, 300-361) */
static struct {
	int iters;
	float dt, under_relax, vel_damping, stiffness_scale, inv_mass_scale, dist_compliance, shape_compliance,
		shape_blend, angle_compliance, angle_blend;
	int use_distance, use_shape, use_angle, use_volume, shape_robust;
	float vol_compliance, vol_aniso;
	int ring_k, max_members, leader_min_hop, member_select, topo_dirty;
	int dist_gs, vol_gs, warp_mode;
	int sc_enabled, sc_within;
	float sc_radius_scale, sc_exclude_scale, sc_search_scale, sc_fast_rel;
	int ground_on;
	float ground_n[3], ground_h, ground_fric, ground_rest, ground_radius, ground_slop, ground_gravity;
	int obj_min_component;
	float obj_shape;
	int jstats;
	kin_t kin[MAX_KIN];
	int kin_count;
	float kin_margin, kin_friction;
	int kin_hits[MAX_KIN];
	float kin_push[MAX_KIN * KIN_ACC];
	int threads;
} P = {
	20, 1.0f / 60.0f, 0.6f, 0.59f, 1.0f, 1.0f, 1e-3f, 0.0f, 0.1f, 0.0f, 0.2f,
	1, 0, 0, 0, 1,
	1e-6f, 0.05f,
	1, 64, 1, 1, 0,
	0, 0, 0,
	0, 0, 1.5f, 2.0f, 1.5f, 0.0f,
	0, { 0.0f, 0.0f, 1.0f }, 0.0f, 0.5f, 0.3f, 0.0f, 0.0f, 0.0f,
	50, 0.0f,
	1,
};

static int fail(const char* msg)
{
	snprintf(S.err, sizeof(S.err), "%s", msg);
	return -1;
}

#define FREE(p) do { free(p); (p) = NULL; } while (0)

static void free_state(void)
{
	FREE(S.off); FREE(S.cnt); FREE(S.nbr); FREE(S.ndist); FREE(S.nstiff);
	FREE(S.pos_curr); FREE(S.pos_next); FREE(S.pos_tmp); FREE(S.pos_rest); FREE(S.vel);
	FREE(S.inv_mass); FREE(S.density); FREE(S.lam_a); FREE(S.lam_b); FREE(S.cm_time); FREE(S.cm_time_next);
	FREE(S.obj_c0); FREE(S.obj_params); FREE(S.obj_disp); FREE(S.obj_boxes); FREE(S.obj_w); FREE(S.obj_q);
	FREE(S.obj_sumq); FREE(S.obj_shift); FREE(S.obj_count); FREE(S.obj_accum); FREE(S.sc_act);
	S.obj_cache = 0; S.obj_shift_valid = 0;
	FREE(S.vol_off); FREE(S.vol_cnt); FREE(S.vol_idx); FREE(S.rev_off); FREE(S.rev_cnt); FREE(S.rev_idx);
	FREE(S.sigma_rest); FREE(S.det_rest); FREE(S.v_rest); FREE(S.rest_len); FREE(S.lam_vol); FREE(S.mat_type);
	FREE(S.cl_c); FREE(S.cl_sinv); FREE(S.cl_coef); FREE(S.vol_gs_order); FREE(S.vol_gs_color_off);
	FREE(S.gs_edge); FREE(S.gs_rest); FREE(S.gs_stiff); FREE(S.gs_lam); FREE(S.gs_color_off);
	FREE(S.inv_mass_saved);
	FREE(S.sc_keys); FREE(S.sc_keys_sorted); FREE(S.sc_idx_sorted); FREE(S.sc_cell_start); FREE(S.sc_cell_end);
	FREE(S.sc_contact); FREE(S.sc_count); FREE(S.sc_dp); FREE(S.sc_dp_cross); FREE(S.obj_id);
	S.built = 0;
	S.att_active = 0;
	S.sc_table = 0;
	S.sc_spacing = 0.0f;
	S.obj_k = 0;
	S.gs_nedges = S.gs_ncolors = 0;
	S.vol_gs_ncolors = S.vol_gs_clusters = 0;
}

static void free_all(void)
{
	free_state();
	/* free_all of xpbd_capi.cu:55-56: contact shapes off with the scene */
	FREE(S.contact_M); FREE(S.contact_rmax); FREE(S.contact_rg);
	S.contact_on = S.contact_col = S.contact_ground = 0;
	S.contact_n = 0;
	FREE(S.pos_in); FREE(S.scales); FREE(S.rots); FREE(S.opacity);
	FREE(S.edges); FREE(S.edge_rest); FREE(S.edge_stiff);
	S.n = 0;
	S.n_edges = 0;
	S.created = 0;
	S.stepped = 0;
}

static inline int nthreads(void) { return P.threads > 0 ? P.threads : omp_get_num_procs(); }

/* ------------------------------------------------------------------------- */
/* graph upload: loadGraph (forward.cu:2702-2779)                             */
/* ------------------------------------------------------------------------- */
static void load_graph(void)
{
	const int n = S.n;
	S.cnt = calloc(n, sizeof(int));
	S.off = calloc(n, sizeof(int));
	for (int k = 0; k < S.n_edges; ++k) {
		const int a = S.edges[2 * k], b = S.edges[2 * k + 1];
		if (a < 0 || b < 0 || a >= n || b >= n || a == b) continue;
		S.cnt[a]++; S.cnt[b]++;
	}
	long long total = 0;
	for (int i = 0; i < n; ++i) { S.off[i] = (int)total; total += S.cnt[i]; }
	S.m = (int)total;
	S.nbr = malloc(sizeof(int) * (total > 0 ? total : 1));
	S.ndist = malloc(sizeof(float) * (total > 0 ? total : 1));
	S.nstiff = malloc(sizeof(float) * (total > 0 ? total : 1));
	int* fill = calloc(n, sizeof(int));
	/* tempNeigh[a].emplace_back(b, rl, st); tempNeigh[b].emplace_back(a, rl, st) in edge order */
	for (int k = 0; k < S.n_edges; ++k) {
		const int a = S.edges[2 * k], b = S.edges[2 * k + 1];
		if (a < 0 || b < 0 || a >= n || b >= n || a == b) continue;
		int ea = S.off[a] + fill[a]++;
		S.nbr[ea] = b; S.ndist[ea] = S.edge_rest[k]; S.nstiff[ea] = S.edge_stiff[k];
		int eb = S.off[b] + fill[b]++;
		S.nbr[eb] = a; S.ndist[eb] = S.edge_rest[k]; S.nstiff[eb] = S.edge_stiff[k];
	}
	free(fill);
}

/* ------------------------------------------------------------------------- */
/* distance GS edges + greedy edge colouring (forward.cu:10407-10517)         */
/* ------------------------------------------------------------------------- */
typedef struct { int a, b; float rest, stiff; int dup; } gsedge_t;
static int cmp_gsedge(const void* x, const void* y)
{
	const gsedge_t* p = x;
	const gsedge_t* q = y;
	if (p->a != q->a) return p->a < q->a ? -1 : 1;
	if (p->b != q->b) return p->b < q->b ? -1 : 1;
	return 0;
}

static void build_distance_gs(void)
{
	const int n = S.n;
	FREE(S.gs_edge); FREE(S.gs_rest); FREE(S.gs_stiff); FREE(S.gs_lam); FREE(S.gs_color_off);
	S.gs_nedges = S.gs_ncolors = 0;
	if (n <= 0 || S.m <= 0) return;
	gsedge_t* dir = malloc(sizeof(gsedge_t) * S.m);
	int nd = 0;
	for (int i = 0; i < n; ++i)
		for (int k = 0; k < S.cnt[i]; ++k) {
			const int e = S.off[i] + k;
			if (e < 0 || e >= S.m) break;
			const int j = S.nbr[e];
			if (j < 0 || j >= n || j == i) continue;
			gsedge_t g = { i < j ? i : j, i < j ? j : i, S.ndist[e], S.nstiff[e], 1 };
			dir[nd++] = g;
		}
	qsort(dir, nd, sizeof(gsedge_t), cmp_gsedge);
	gsedge_t* und = malloc(sizeof(gsedge_t) * (nd > 0 ? nd : 1));
	int E = 0;
	for (int t = 0; t < nd; ++t) {
		if (E > 0 && und[E - 1].a == dir[t].a && und[E - 1].b == dir[t].b) {
			und[E - 1].rest += dir[t].rest;
			und[E - 1].stiff += dir[t].stiff;
			und[E - 1].dup++;
		}
		else und[E++] = dir[t];
	}
	free(dir);
	for (int e = 0; e < E; ++e) {
		und[e].rest /= (float)und[e].dup;
		und[e].stiff /= (float)und[e].dup;
	}
	if (E == 0) { free(und); return; }
	int* deg = calloc(n, sizeof(int));
	for (int e = 0; e < E; ++e) { deg[und[e].a]++; deg[und[e].b]++; }
	int maxDeg = 0;
	for (int i = 0; i < n; ++i) if (deg[i] > maxDeg) maxDeg = deg[i];
	free(deg);
	const int words = (2 * maxDeg + 63) / 64;
	uint64_t* used = calloc((size_t)n * words, sizeof(uint64_t));
	int* color = malloc(sizeof(int) * E);
	int numColors = 0;
	for (int e = 0; e < E; ++e) {
		uint64_t* ua = &used[(size_t)und[e].a * words];
		uint64_t* ub = &used[(size_t)und[e].b * words];
		int c = -1;
		for (int w = 0; w < words && c < 0; ++w) {
			const uint64_t freeBits = ~(ua[w] | ub[w]);
			if (!freeBits) continue;
			int bit = 0;
			while (!((freeBits >> bit) & 1ull)) ++bit;
			c = w * 64 + bit;
		}
		ua[c >> 6] |= 1ull << (c & 63);
		ub[c >> 6] |= 1ull << (c & 63);
		color[e] = c;
		if (c + 1 > numColors) numColors = c + 1;
	}
	free(used);
	S.gs_color_off = calloc(numColors + 1, sizeof(int));
	for (int e = 0; e < E; ++e) S.gs_color_off[color[e] + 1]++;
	for (int c = 0; c < numColors; ++c) S.gs_color_off[c + 1] += S.gs_color_off[c];
	int* fill = malloc(sizeof(int) * (numColors > 0 ? numColors : 1));
	memcpy(fill, S.gs_color_off, sizeof(int) * numColors);
	S.gs_edge = malloc(sizeof(int) * 2 * (size_t)E);
	S.gs_rest = malloc(sizeof(float) * (size_t)E);
	S.gs_stiff = malloc(sizeof(float) * (size_t)E);
	S.gs_lam = calloc((size_t)E, sizeof(float));
	for (int e = 0; e < E; ++e) {
		const int p = fill[color[e]]++;
		S.gs_edge[2 * p] = und[e].a;
		S.gs_edge[2 * p + 1] = und[e].b;
		S.gs_rest[p] = und[e].rest;
		S.gs_stiff[p] = und[e].stiff;
	}
	free(fill); free(color); free(und);
	S.gs_nedges = E;
	S.gs_ncolors = numColors;
}

/* ------------------------------------------------------------------------- */
/* volume clusters: rebuildVolumeClusters (forward.cu:9814-10403)             */
/* ------------------------------------------------------------------------- */
typedef struct { int* v; int n, cap; } ivec;
static inline void iv_push(ivec* a, int x)
{
	if (a->n == a->cap) { a->cap = a->cap ? 2 * a->cap : 16; a->v = realloc(a->v, sizeof(int) * a->cap); }
	a->v[a->n++] = x;
}

#define HARD_CAP 8192
static inline float dist2f(f3 a, f3 b)
{
	const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
	return dx * dx + dy * dy + dz * dz;
}

/* computeMembers (forward.cu:9871-10033) with member select 1 (farthest point, 9994-10026) or
 * 0 (stride, 10027-10031).  The result replaces *out. */
static void compute_members(int i, int* stamp, ivec* frontier, ivec* next, ivec* col, float* md, char* taken,
	ivec* out)
{
	const int n = S.n, k = P.ring_k, cap = P.max_members;
	col->n = 0;
	if (k <= 1) {
		for (int e = 0; e < S.cnt[i]; ++e) {
			const int j = S.nbr[S.off[i] + e];
			if (j >= 0 && j < n && j != i) iv_push(col, j);
		}
	}
	else {
		frontier->n = 0;
		stamp[i] = i;
		iv_push(frontier, i);
		for (int d = 0; d < k && frontier->n > 0 && col->n < HARD_CAP; ++d) {
			next->n = 0;
			int capped = 0;
			for (int fi = 0; fi < frontier->n; ++fi) {
				const int f = frontier->v[fi];
				for (int e = 0; e < S.cnt[f]; ++e) {
					const int j = S.nbr[S.off[f] + e];
					if (j < 0 || j >= n || stamp[j] == i) continue;
					stamp[j] = i;
					iv_push(col, j);
					iv_push(next, j);
					if (col->n >= HARD_CAP) { capped = 1; break; }
				}
				if (capped) break;
			}
			ivec t = *frontier; *frontier = *next; *next = t;
			if (capped) break;
		}
	}
	out->n = 0;
	if (col->n <= cap) {
		for (int t = 0; t < col->n; ++t) iv_push(out, col->v[t]);
		return;
	}
	if (P.member_select == 1) {
		const f3 cpos = S.pos_rest[i];
		const int Mc = col->n;
		int cur = 0;
		float best = -1.0f;
		for (int m = 0; m < Mc; ++m) {
			const float dd = dist2f(S.pos_rest[col->v[m]], cpos);
			md[m] = dd;
			taken[m] = 0;
			if (dd > best) { best = dd; cur = m; }
		}
		for (int s = 0; s < cap; ++s) {
			taken[cur] = 1;
			iv_push(out, col->v[cur]);
			const f3 cp = S.pos_rest[col->v[cur]];
			int nxt = -1;
			float nbest = -1.0f;
			for (int m = 0; m < Mc; ++m) {
				if (taken[m]) continue;
				const float dd = dist2f(S.pos_rest[col->v[m]], cp);
				if (dd < md[m]) md[m] = dd;
				if (md[m] > nbest) { nbest = md[m]; nxt = m; }
			}
			if (nxt < 0) break;
			cur = nxt;
		}
	}
	else {
		const double stride = (double)col->n / (double)cap;
		for (int t = 0; t < cap; ++t) iv_push(out, col->v[(size_t)(t * stride)]);
	}
}

/* precomputeVolumeGaussianKernel (forward.cu:7691-7844), mixture rest off (forward.cu:393) */
static void precompute_volume_node(int idx)
{
	const int N = S.n;
	float* sig = S.sigma_rest + (size_t)idx * 6;
	for (int k = 0; k < 6; ++k) sig[k] = 0.0f;
	S.det_rest[idx] = 0.0f;
	S.v_rest[idx] = 0.0f;
	S.mat_type[idx] = 3;
	{
		const f3 p0g = S.pos_rest[idx];
		const int goff = S.off[idx], gcnt = S.cnt[idx];
		float dmin = FLT_MAX;
		for (int e = 0; e < gcnt; ++e) {
			const int j = S.nbr[goff + e];
			if (j < 0 || j >= N || j == idx) continue;
			const float dl = f3_len(f3_sub(S.pos_rest[j], p0g));
			if (dl > 1e-12f) dmin = fminf(dmin, dl);
		}
		S.rest_len[idx] = (dmin < FLT_MAX) ? dmin : 0.0f;
	}
	const int off = S.vol_off[idx], cnt = S.vol_cnt[idx];
	if (cnt < 4) return;
	const f3 p0 = S.pos_rest[idx];
	f3 c = p0;
	int used = 0;
	for (int k = 0; k < cnt; ++k) {
		const int j = S.vol_idx[off + k];
		if (j < 0 || j >= N) continue;
		c = f3_add(c, S.pos_rest[j]);
		++used;
	}
	if (used < 3) return;
	const float n = (float)(used + 1);
	const float invN = 1.0f / n;
	c = f3_mul(c, invN);
	m3 Sm = m3_zero();
	{
		const f3 d = f3_sub(S.pos_rest[idx], c);
		m3_add_outer(&Sm, d, d);
	}
	for (int k = 0; k < cnt; ++k) {
		const int j = S.vol_idx[off + k];
		if (j < 0 || j >= N) continue;
		const f3 d = f3_sub(S.pos_rest[j], c);
		m3_add_outer(&Sm, d, d);
	}
	Sm = m3_scale(&Sm, invN);
	float sRest, detHatRest;
	if (!sigma_scale_det(&Sm, &sRest, &detHatRest)) { S.mat_type[idx] = 4; return; }
	f3 eig;
	m3 V;
	eig_glm(&Sm, &eig, &V);
	const float lmax = fmaxf(eig.z, 1e-24f);
	const float a1 = eig.x / lmax, a2 = eig.y / lmax;
	if (a1 > P.vol_aniso) S.mat_type[idx] = 0;
	else if (a2 > P.vol_aniso) S.mat_type[idx] = 1;
	else S.mat_type[idx] = 2;
	store_sym3(sig, &Sm);
	const float d = sRest * sRest * sRest * detHatRest;
	S.det_rest[idx] = d;
	S.v_rest[idx] = (4.0f / 3.0f) * 3.14159265f * sqrtf(fmaxf(d, 0.0f));
}

/* buildVolumeGSColors (forward.cu:9745-9812) */
static void build_volume_gs_colors(ivec* members, const char* isLeader)
{
	const int N = S.n;
	FREE(S.vol_gs_order); FREE(S.vol_gs_color_off);
	S.vol_gs_ncolors = S.vol_gs_clusters = 0;
	double work = 0.0;
	for (int j = 0; j < N; ++j) work += (double)S.rev_cnt[j] * S.rev_cnt[j];
	int M = 0;
	for (int i = 0; i < N; ++i) if (isLeader[i]) ++M;
	if (M == 0 || work > 4.0e9) return;
	int* color = malloc(sizeof(int) * N);
	for (int i = 0; i < N; ++i) color[i] = -1;
	int stampCap = 64, numColors = 0;
	int* stamp = malloc(sizeof(int) * stampCap);
	for (int l = 0; l < N; ++l) {
		if (!isLeader[l]) continue;
		if (stampCap < numColors + 1) {
			stamp = realloc(stamp, sizeof(int) * (numColors + 1) * 2);
			for (int c = stampCap; c < (numColors + 1) * 2; ++c) stamp[c] = -1;
			stampCap = (numColors + 1) * 2;
		}
		if (l == 0 || numColors == 0) {
			/* first use: initialise any untouched slots */
		}
#define FORBID(jj)                                                           \
	do {                                                                     \
		const int j_ = (jj);                                                 \
		for (int q = 0; q < S.rev_cnt[j_]; ++q) {                            \
			const int mm = S.rev_idx[S.rev_off[j_] + q];                     \
			if (mm >= 0 && mm < N && color[mm] >= 0) stamp[color[mm]] = l;  \
		}                                                                    \
	} while (0)
		FORBID(l);
		for (int t = 0; t < members[l].n; ++t) {
			const int j = members[l].v[t];
			if (j >= 0 && j < N) FORBID(j);
		}
#undef FORBID
		int c = 0;
		while (c < numColors && stamp[c] == l) ++c;
		color[l] = c;
		if (c + 1 > numColors) numColors = c + 1;
	}
	free(stamp);
	S.vol_gs_color_off = calloc(numColors + 1, sizeof(int));
	for (int l = 0; l < N; ++l) if (isLeader[l]) S.vol_gs_color_off[color[l] + 1]++;
	for (int c = 0; c < numColors; ++c) S.vol_gs_color_off[c + 1] += S.vol_gs_color_off[c];
	int* fill = malloc(sizeof(int) * (numColors > 0 ? numColors : 1));
	memcpy(fill, S.vol_gs_color_off, sizeof(int) * numColors);
	S.vol_gs_order = malloc(sizeof(int) * M);
	for (int l = 0; l < N; ++l) if (isLeader[l]) S.vol_gs_order[fill[color[l]]++] = l;
	free(fill);
	free(color);
	S.vol_gs_ncolors = numColors;
	S.vol_gs_clusters = M;
}

static void rebuild_volume_clusters(void)
{
	const int N = S.n;
	if (N <= 0) return;
	const int leaderR = P.leader_min_hop > 1 ? P.leader_min_hop : 1;
	char* isLeader = calloc(N, 1);
	ivec* members = calloc(N, sizeof(ivec));
	int* coverCnt = calloc(N, sizeof(int));
	if (leaderR <= 1) {
		/* r = 1: every node leads its own cluster (forward.cu:10047-10069) */
		memset(isLeader, 1, N);
		S.leader_count = N;
#pragma omp parallel num_threads(nthreads())
		{
			int* stamp = malloc(sizeof(int) * N);
			for (int t = 0; t < N; ++t) stamp[t] = -1;
			ivec fr = { 0 }, nx = { 0 }, col = { 0 };
			float* md = malloc(sizeof(float) * HARD_CAP);
			char* taken = malloc(HARD_CAP);
#pragma omp for schedule(dynamic, 512)
			for (int i = 0; i < N; ++i) compute_members(i, stamp, &fr, &nx, &col, md, taken, &members[i]);
			free(stamp); free(md); free(taken); free(fr.v); free(nx.v); free(col.v);
		}
	}
	else {
		/* r >= 2: greedy cover (forward.cu:10070-10132) */
		const int targetCover = leaderR < 6 ? leaderR : 6;
		int* stamp = malloc(sizeof(int) * N);
		int* stampR = malloc(sizeof(int) * N);
		for (int t = 0; t < N; ++t) { stamp[t] = -1; stampR[t] = -1; }
		ivec fr = { 0 }, nx = { 0 }, col = { 0 };
		float* md = malloc(sizeof(float) * HARD_CAP);
		char* taken = malloc(HARD_CAP);
		int leaderCnt = 0;
		for (int seed = 0; seed < N; ++seed) {
			if (coverCnt[seed] >= targetCover) continue;
			if (stampR[seed] == -2) continue;
			isLeader[seed] = 1;
			++leaderCnt;
			compute_members(seed, stamp, &fr, &nx, &col, md, taken, &members[seed]);
			++coverCnt[seed];
			for (int t = 0; t < members[seed].n; ++t) {
				const int j = members[seed].v[t];
				if (j >= 0 && j < N) ++coverCnt[j];
			}
			fr.n = 0;
			stampR[seed] = -2;
			iv_push(&fr, seed);
			for (int d = 0; d < leaderR - 1 && fr.n > 0; ++d) {
				nx.n = 0;
				for (int fi = 0; fi < fr.n; ++fi) {
					const int f = fr.v[fi];
					for (int e = 0; e < S.cnt[f]; ++e) {
						const int j = S.nbr[S.off[f] + e];
						if (j < 0 || j >= N || stampR[j] == -2) continue;
						stampR[j] = -2;
						iv_push(&nx, j);
					}
				}
				ivec t2 = fr; fr = nx; nx = t2;
			}
		}
		int progressed = 1;
		while (progressed) {
			progressed = 0;
			for (int i = 0; i < N; ++i) {
				if (coverCnt[i] >= targetCover) continue;
				if (isLeader[i]) continue;
				isLeader[i] = 1;
				++leaderCnt;
				compute_members(i, stamp, &fr, &nx, &col, md, taken, &members[i]);
				++coverCnt[i];
				for (int t = 0; t < members[i].n; ++t) {
					const int j = members[i].v[t];
					if (j >= 0 && j < N) ++coverCnt[j];
				}
				progressed = 1;
			}
		}
		S.leader_count = leaderCnt;
		free(stamp); free(stampR); free(md); free(taken); free(fr.v); free(nx.v); free(col.v);
	}
	free(coverCnt);
	/* CSR flatten (forward.cu:10160-10200) */
	FREE(S.vol_off); FREE(S.vol_cnt); FREE(S.vol_idx); FREE(S.rev_off); FREE(S.rev_cnt); FREE(S.rev_idx);
	S.vol_off = malloc(sizeof(int) * N);
	S.vol_cnt = malloc(sizeof(int) * N);
	long long total = 0;
	for (int i = 0; i < N; ++i) { S.vol_off[i] = (int)total; S.vol_cnt[i] = members[i].n; total += members[i].n; }
	S.vol_total = total;
	S.vol_idx = malloc(sizeof(int) * (total > 0 ? total : 1));
	for (int i = 0; i < N; ++i)
		if (members[i].n > 0) memcpy(S.vol_idx + S.vol_off[i], members[i].v, sizeof(int) * members[i].n);
	/* transposed CSR with self entries for leaders (forward.cu:10204-10246) */
	S.rev_cnt = calloc(N, sizeof(int));
	for (int i = 0; i < N; ++i) if (isLeader[i]) ++S.rev_cnt[i];
	for (int i = 0; i < N; ++i)
		for (int t = 0; t < members[i].n; ++t) ++S.rev_cnt[members[i].v[t]];
	S.rev_off = malloc(sizeof(int) * N);
	long long revTotal = 0;
	for (int i = 0; i < N; ++i) { S.rev_off[i] = (int)revTotal; revTotal += S.rev_cnt[i]; }
	S.rev_total = revTotal;
	S.rev_idx = malloc(sizeof(int) * (revTotal > 0 ? revTotal : 1));
	int* cursor = malloc(sizeof(int) * N);
	memcpy(cursor, S.rev_off, sizeof(int) * N);
	for (int i = 0; i < N; ++i) if (isLeader[i]) S.rev_idx[cursor[i]++] = i;
	for (int i = 0; i < N; ++i)
		for (int t = 0; t < members[i].n; ++t) S.rev_idx[cursor[members[i].v[t]]++] = i;
	free(cursor);
	build_volume_gs_colors(members, isLeader);
	S.avg_members = S.leader_count > 0 ? (float)((double)total / S.leader_count) : 0.0f;
	/* rest covariance (forward.cu:10264-10281) */
#pragma omp parallel for schedule(static) num_threads(nthreads())
	for (int i = 0; i < N; ++i) precompute_volume_node(i);
	memset(S.lam_vol, 0, sizeof(float) * N);
	for (int i = 0; i < N; ++i) free(members[i].v);
	free(members);
	free(isLeader);
}

/* ------------------------------------------------------------------------- */
/* ensureChainmailGPU (forward.cu:10519-10845)                                */
/* ------------------------------------------------------------------------- */
static void ensure_built(void)
{
	if (S.built) {
		if (P.topo_dirty) {
			P.topo_dirty = 0;
			rebuild_volume_clusters();
		}
		return;
	}
	free_state();
	const int N = S.n;
	load_graph();
	S.pos_curr = malloc(sizeof(f3) * N);
	S.pos_next = malloc(sizeof(f3) * N);
	S.pos_tmp = malloc(sizeof(f3) * N);
	S.pos_rest = malloc(sizeof(f3) * N);
	S.vel = calloc(N, sizeof(f3));
	S.inv_mass = malloc(sizeof(float) * N);
	S.density = malloc(sizeof(float) * N);
	for (int i = 0; i < N; ++i) {
		S.pos_curr[i] = S.pos_rest[i] = mk3(S.pos_in[3 * i], S.pos_in[3 * i + 1], S.pos_in[3 * i + 2]);
		S.inv_mass[i] = 1.0f;
		S.density[i] = S.opacity[i];
	}
	S.cm_time = malloc(sizeof(float) * N);
	S.cm_time_next = malloc(sizeof(float) * N);
	for (int i = 0; i < N; ++i) S.cm_time[i] = 1e9f;
	const int M = S.m > 0 ? S.m : 1;
	S.lam_a = calloc(M, sizeof(float));
	S.lam_b = calloc(M, sizeof(float));
	S.sigma_rest = calloc((size_t)6 * N, sizeof(float));
	S.det_rest = calloc(N, sizeof(float));
	S.v_rest = calloc(N, sizeof(float));
	S.rest_len = calloc(N, sizeof(float));
	S.mat_type = calloc(N, sizeof(int));
	S.lam_vol = calloc(N, sizeof(float));
	S.cl_c = calloc(N, sizeof(f3));
	S.cl_sinv = calloc((size_t)6 * N, sizeof(float));
	S.cl_coef = calloc(N, sizeof(float));
	build_distance_gs();
	P.topo_dirty = 0;
	rebuild_volume_clusters();
	S.built = 1;
}

/* ------------------------------------------------------------------------- */
/* per-iteration kernels                                                      */
/* ------------------------------------------------------------------------- */
/* xpbdPredictKernel (forward.cu:5954-5979) */
static void predict(f3 gravity, float dt)
{
#pragma omp parallel for schedule(static) num_threads(nthreads())
	for (int i = 0; i < S.n; ++i) {
		const f3 x = S.pos_curr[i];
		f3 v = S.vel[i];
		if (S.inv_mass[i] > 0.0f) {
			v = f3_add(v, f3_mul(gravity, dt));
			S.pos_next[i] = f3_add(x, f3_mul(v, dt));
			S.vel[i] = v;
		}
		else {
			S.pos_next[i] = x;
			S.vel[i] = mk3(0.0f, 0.0f, 0.0f);
		}
	}
}

/* xpbdSolveJacobiKernel (forward.cu:6484-6571) */
static void distance_jacobi(const f3* pin, f3* pout, const float* lin, float* lout, float dt)
{
	const int N = S.n;
	const float ims = P.inv_mass_scale, ss = P.stiffness_scale, ur = P.under_relax, gc = P.dist_compliance;
#pragma omp parallel for schedule(static) num_threads(nthreads())
	for (int idx = 0; idx < N; ++idx) {
		const f3 pi = pin[idx];
		const float wi = S.inv_mass[idx] * ims;
		f3 accum = mk3(0, 0, 0);
		int validCount = 0;
		const int off = S.off[idx], cnt = S.cnt[idx];
		const float dt2 = fmaxf(dt * dt, 1e-8f);
		for (int k = 0; k < cnt; ++k) {
			const int edge = off + k;
			const int j = S.nbr[edge];
			float lambda = lin[edge];
			if (j < 0 || j >= N) { lout[edge] = lambda; continue; }
			const f3 pj = pin[j];
			const f3 diff = f3_sub(pi, pj);
			const float d = f3_len(diff);
			if (d < 1e-7f) { lout[edge] = lambda; continue; }
			const float L0 = S.ndist[edge];
			const float C = d - L0;
			const f3 grad = f3_mul(diff, 1.0f / d);
			const float wj = S.inv_mass[j] * ims;
			const float stiff = fmaxf(S.nstiff[edge] * ss, 1e-6f);
			const float alpha = gc / stiff;
			const float alpha_tilde = alpha / dt2;
			const float denom = (wi + wj) + alpha_tilde;
			if (denom < 1e-8f) { lout[edge] = lambda; continue; }
			const float delta_lambda = (-C - alpha_tilde * lambda) / denom;
			lambda += delta_lambda;
			lout[edge] = lambda;
			if (wi > 0.0f) {
				accum = f3_add(accum, f3_mul(grad, wi * delta_lambda));
				validCount++;
			}
		}
		f3 outPos = pi;
		if (wi > 0.0f && validCount > 0) {
			const f3 avg = f3_mul(accum, 1.0f / (float)validCount);
			outPos = f3_add(pi, f3_mul(avg, ur));
		}
		pout[idx] = outPos;
	}
}

/* xpbdDistanceGSColorKernel (forward.cu:6576-6621), one colour sequentially (edges of a
 * colour share no vertex, so order inside a colour does not matter) */
static void distance_gs(f3* pos, float dt)
{
	const float ims = P.inv_mass_scale, ss = P.stiffness_scale, gc = P.dist_compliance;
	for (int c = 0; c < S.gs_ncolors; ++c) {
		const int begin = S.gs_color_off[c], end = S.gs_color_off[c + 1];
#pragma omp parallel for schedule(static) num_threads(nthreads())
		for (int e = begin; e < end; ++e) {
			const int a = S.gs_edge[2 * e], b = S.gs_edge[2 * e + 1];
			if (a < 0 || a >= S.n || b < 0 || b >= S.n) continue;
			const float wi = S.inv_mass[a] * ims, wj = S.inv_mass[b] * ims;
			if (wi + wj <= 0.0f) continue;
			const f3 pi = pos[a], pj = pos[b];
			const f3 diff = f3_sub(pi, pj);
			const float d = f3_len(diff);
			if (d < 1e-7f) continue;
			const float dt2 = fmaxf(dt * dt, 1e-8f);
			const float s = fmaxf(S.gs_stiff[e] * ss, 1e-6f);
			const float alpha_tilde = (gc / s) / dt2;
			const float denom = (wi + wj) + alpha_tilde;
			if (denom < 1e-8f) continue;
			const float C = d - S.gs_rest[e];
			const float lam = S.gs_lam[e];
			const float delta_lambda = (-C - alpha_tilde * lam) / denom;
			S.gs_lam[e] = lam + delta_lambda;
			const f3 nn = f3_mul(diff, 1.0f / d);
			if (wi > 0.0f) pos[a] = f3_add(pi, f3_mul(nn, wi * delta_lambda));
			if (wj > 0.0f) pos[b] = f3_sub(pj, f3_mul(nn, wj * delta_lambda));
		}
	}
}

static inline int vol_use_warp(void)
{
	if (P.warp_mode == 2) return 1;
	if (P.warp_mode == 1) return 0;
	return S.avg_members >= 40.0f;
}

/* Step 2-5 of the cluster solve shared by the thread and warp kernels
 * (forward.cu:8583-8650 / 8780-8812): J, Sigma^-1.  Returns 0 when the cluster is skipped. */
static int cluster_j_sinv(const m3* Scur, float detRest, float* Jout, float* Cout, m3* Sinv)
{
	float sCur, detHatCur;
	if (!sigma_scale_det(Scur, &sCur, &detHatCur)) return 0;
	const float detCur = sCur * sCur * sCur * detHatCur;
	if (detRest < 1e-30f) return 0;
	float J = sqrtf(detCur / detRest);
	if (!isfinite(J) || J <= 0.0f) return 0;
	if (J > 3.0f || J < 0.333f) J = fminf(3.0f, fmaxf(0.333f, J));
	const float C = J - 1.0f;
	if (fabsf(C) < 1e-4f) return 0;
	m3 Sreg = *Scur;
	if (detHatCur < 0.2f) {
		const float d = 0.06f * sCur;
		Sreg.m[0][0] += d; Sreg.m[1][1] += d; Sreg.m[2][2] += d;
	}
	if (!inverse3x3_safe(&Sreg, Sinv, 1e-20f)) return 0;
	*Jout = J;
	*Cout = C;
	return 1;
}

/* Step 5-6: delta lambda and the blackboard write (forward.cu:8637-8663 / 8837-8862) */
static void cluster_commit(int idx, float denom, float C, float gs, f3 c, const m3* Sinv, float dt)
{
	const float dt2 = fmaxf(dt * dt, 1e-8f);
	const float alphaT = P.vol_compliance / dt2;
	const float den = denom + alphaT;
	if (!(den > 1e-12f)) { S.cl_coef[idx] = 0.0f; return; }
	const float lam = S.lam_vol[idx];
	const float dLam = (-C - alphaT * lam) / den;
	if (!isfinite(dLam)) { S.cl_coef[idx] = 0.0f; return; }
	S.lam_vol[idx] = lam + dLam;
	S.cl_c[idx] = c;
	store_sym3(S.cl_sinv + (size_t)idx * 6, Sinv);
	S.cl_coef[idx] = dLam * gs;
}

/* xpbdVolumeClusterSolveKernel (forward.cu:8531-8664), one thread per cluster */
static void cluster_solve_thread(int idx, const f3* pin, float dt)
{
	const int N = S.n;
	const float ims = P.inv_mass_scale;
	S.cl_coef[idx] = 0.0f;
	const f3 pi = pin[idx];
	if (S.mat_type[idx] != 0) return;
	const int off = S.vol_off[idx], cnt = S.vol_cnt[idx];
	f3 c = pi;
	int used = 0;
	for (int k = 0; k < cnt; ++k) {
		const int j = S.vol_idx[off + k];
		if (j < 0 || j >= N) continue;
		c = f3_add(c, pin[j]);
		++used;
	}
	if (used < 3) return;
	const float n = (float)(used + 1);
	const float invN = 1.0f / n;
	c = f3_mul(c, invN);
	m3 Scur = m3_zero();
	{
		const f3 d = f3_sub(pi, c);
		m3_add_outer(&Scur, d, d);
	}
	for (int k = 0; k < cnt; ++k) {
		const int j = S.vol_idx[off + k];
		if (j < 0 || j >= N) continue;
		const f3 d = f3_sub(pin[j], c);
		m3_add_outer(&Scur, d, d);
	}
	Scur = m3_scale(&Scur, invN);
	float J, C;
	m3 Sinv;
	if (!cluster_j_sinv(&Scur, S.det_rest[idx], &J, &C, &Sinv)) return;
	const float gs = J * invN;
	float denom = 0.0f;
	{
		const f3 g = f3_mul(m3_mulv(&Sinv, f3_sub(pi, c)), gs);
		denom += (S.inv_mass[idx] * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
	}
	for (int k = 0; k < cnt; ++k) {
		const int j = S.vol_idx[off + k];
		if (j < 0 || j >= N) continue;
		const f3 g = f3_mul(m3_mulv(&Sinv, f3_sub(pin[j], c)), gs);
		denom += (S.inv_mass[j] * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
	}
	cluster_commit(idx, denom, C, gs, c, &Sinv, dt);
}

/* xpbdVolumeClusterSolveWarpKernel (forward.cu:8702-8863): lane-strided members, butterfly sums.
 * The 8-slot register cache does not change the arithmetic, only where positions come from. */
static void cluster_solve_warp(int idx, const f3* pin, float dt)
{
	const int N = S.n;
	const float ims = P.inv_mass_scale;
	if (S.mat_type[idx] != 0) { S.cl_coef[idx] = 0.0f; return; }
	const int off = S.vol_off[idx], cnt = S.vol_cnt[idx];
	const f3 pi = pin[idx];
	float lx[32], ly[32], lz[32], lc[32];
	for (int L = 0; L < 32; ++L) {
		f3 psum = mk3(0, 0, 0);
		int ucnt = 0;
		for (int k = L; k < cnt; k += 32) {
			const int j = S.vol_idx[off + k];
			if (j < 0 || j >= N) continue;
			psum = f3_add(psum, pin[j]);
			++ucnt;
		}
		lx[L] = psum.x; ly[L] = psum.y; lz[L] = psum.z; lc[L] = (float)ucnt;
	}
	const float sx = warp_allsum(lx), sy = warp_allsum(ly), sz = warp_allsum(lz);
	const int used = (int)(warp_allsum(lc) + 0.5f);
	if (used < 3) { S.cl_coef[idx] = 0.0f; return; }
	const float n = (float)(used + 1);
	const float invN = 1.0f / n;
	const f3 c = mk3((sx + pi.x) * invN, (sy + pi.y) * invN, (sz + pi.z) * invN);
	float a[6][32];
	for (int L = 0; L < 32; ++L) {
		float a00 = 0.f, a11 = 0.f, a22 = 0.f, a01 = 0.f, a02 = 0.f, a12 = 0.f;
		for (int k = L; k < cnt; k += 32) {
			const int j = S.vol_idx[off + k];
			if (j < 0 || j >= N) continue;
			const f3 p = pin[j];
			const float dx = p.x - c.x, dy = p.y - c.y, dz = p.z - c.z;
			a00 += dx * dx; a11 += dy * dy; a22 += dz * dz;
			a01 += dx * dy; a02 += dx * dz; a12 += dy * dz;
		}
		if (L == 0) {
			const float dx = pi.x - c.x, dy = pi.y - c.y, dz = pi.z - c.z;
			a00 += dx * dx; a11 += dy * dy; a22 += dz * dz;
			a01 += dx * dy; a02 += dx * dz; a12 += dy * dz;
		}
		a[0][L] = a00; a[1][L] = a11; a[2][L] = a22; a[3][L] = a01; a[4][L] = a02; a[5][L] = a12;
	}
	m3 Scur = m3_zero();
	Scur.m[0][0] = warp_allsum(a[0]) * invN;
	Scur.m[1][1] = warp_allsum(a[1]) * invN;
	Scur.m[2][2] = warp_allsum(a[2]) * invN;
	const float s01 = warp_allsum(a[3]) * invN, s02 = warp_allsum(a[4]) * invN, s12 = warp_allsum(a[5]) * invN;
	Scur.m[0][1] = Scur.m[1][0] = s01;
	Scur.m[0][2] = Scur.m[2][0] = s02;
	Scur.m[1][2] = Scur.m[2][1] = s12;
	float J, C;
	m3 Sinv;
	if (!cluster_j_sinv(&Scur, S.det_rest[idx], &J, &C, &Sinv)) { S.cl_coef[idx] = 0.0f; return; }
	const float gs = J * invN;
	float ds[32];
	for (int L = 0; L < 32; ++L) {
		float dsum = 0.0f;
		for (int k = L; k < cnt; k += 32) {
			const int j = S.vol_idx[off + k];
			if (j < 0 || j >= N) continue;
			const f3 p = pin[j];
			const f3 g = f3_mul(m3_mulv(&Sinv, mk3(p.x - c.x, p.y - c.y, p.z - c.z)), gs);
			dsum += (S.inv_mass[j] * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
		}
		if (L == 0) {
			const f3 g = f3_mul(m3_mulv(&Sinv, mk3(pi.x - c.x, pi.y - c.y, pi.z - c.z)), gs);
			dsum += (S.inv_mass[idx] * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
		}
		ds[L] = dsum;
	}
	const float denom = warp_allsum(ds);
	cluster_commit(idx, denom, C, gs, c, &Sinv, dt);
}

/* one cluster record applied to node position pi (forward.cu:9212-9222) */
static inline int gather_one(int i, f3 pi, float wi, f3* dp)
{
	const float coef = S.cl_coef[i];
	if (coef == 0.0f) return 0;
	const m3 Sinv = load_sym3(S.cl_sinv + (size_t)i * 6);
	const f3 d = f3_sub(pi, S.cl_c[i]);
	const f3 g = m3_mulv(&Sinv, d);
	*dp = mk3(g.x * wi * coef, g.y * wi * coef, g.z * wi * coef);
	if (!f3_finite(*dp)) return 0;
	return 1;
}

static inline f3 gather_finish(f3 pi, f3 avg, int idx)
{
	const float rl = S.rest_len[idx];
	if (rl > 1e-12f) {
		const float maxStep = 0.25f * rl;
		const float len = f3_len(avg);
		if (len > maxStep && len > 1e-20f) avg = f3_mul(avg, maxStep / len);
	}
	return f3_add(pi, f3_mul(avg, P.under_relax));
}

/* xpbdVolumeGatherApplyKernel (forward.cu:9187-9243) */
static f3 gather_thread(int idx, const f3* pin)
{
	const int N = S.n;
	const f3 pi = pin[idx];
	const float wi = S.inv_mass[idx] * P.inv_mass_scale;
	if (wi <= 0.0f) return pi;
	const int off = S.rev_off[idx], cnt = S.rev_cnt[idx];
	f3 sum = mk3(0, 0, 0);
	int received = 0;
	for (int k = 0; k < cnt; ++k) {
		const int i = S.rev_idx[off + k];
		if (i < 0 || i >= N) continue;
		f3 dp;
		if (!gather_one(i, pi, wi, &dp)) continue;
		sum = f3_add(sum, dp);
		++received;
	}
	if (received <= 0) return pi;
	f3 avg = f3_mul(sum, 1.0f / (float)received);
	if (!f3_finite(avg)) return pi;
	return gather_finish(pi, avg, idx);
}

/* xpbdVolumeGatherApplyWarpKernel (forward.cu:9262-9323) */
static f3 gather_warp(int idx, const f3* pin)
{
	const int N = S.n;
	const f3 pi = pin[idx];
	const float wi = S.inv_mass[idx] * P.inv_mass_scale;
	if (wi <= 0.0f) return pi;
	const int off = S.rev_off[idx], cnt = S.rev_cnt[idx];
	float lx[32], ly[32], lz[32], lc[32];
	for (int L = 0; L < 32; ++L) {
		f3 sum = mk3(0, 0, 0);
		int received = 0;
		for (int k = L; k < cnt; k += 32) {
			const int i = S.rev_idx[off + k];
			if (i < 0 || i >= N) continue;
			f3 dp;
			if (!gather_one(i, pi, wi, &dp)) continue;
			sum = f3_add(sum, dp);
			++received;
		}
		lx[L] = sum.x; ly[L] = sum.y; lz[L] = sum.z; lc[L] = (float)received;
	}
	const float sx = warp_allsum(lx), sy = warp_allsum(ly), sz = warp_allsum(lz);
	const int rec = (int)(warp_allsum(lc) + 0.5f);
	if (rec <= 0) return pi;
	const float invRec = 1.0f / (float)rec;
	f3 avg = mk3(sx * invRec, sy * invRec, sz * invRec);
	if (!f3_finite(avg)) return pi;
	return gather_finish(pi, avg, idx);
}

/* xpbdVolumeGSColorKernel (forward.cu:9041-9183): cluster solve on current positions, then
 * in-place update of every member without averaging */
static void volume_gs(f3* pos, float dt)
{
	const int N = S.n;
	const float ims = P.inv_mass_scale;
	for (int col = 0; col < S.vol_gs_ncolors; ++col) {
		const int begin = S.vol_gs_color_off[col], end = S.vol_gs_color_off[col + 1];
#pragma omp parallel for schedule(static) num_threads(nthreads())
		for (int t = begin; t < end; ++t) {
			const int idx = S.vol_gs_order[t];
			if (idx < 0 || idx >= N) continue;
			if (S.mat_type[idx] != 0) continue;
			const int off = S.vol_off[idx], cnt = S.vol_cnt[idx];
			const f3 pi = pos[idx];
			f3 c = pi;
			int used = 0;
			for (int k = 0; k < cnt; ++k) {
				const int j = S.vol_idx[off + k];
				if (j < 0 || j >= N) continue;
				c = f3_add(c, pos[j]);
				++used;
			}
			if (used < 3) continue;
			const float n = (float)(used + 1);
			const float invN = 1.0f / n;
			c = f3_mul(c, invN);
			m3 Scur = m3_zero();
			{
				const f3 d = f3_sub(pi, c);
				m3_add_outer(&Scur, d, d);
			}
			for (int k = 0; k < cnt; ++k) {
				const int j = S.vol_idx[off + k];
				if (j < 0 || j >= N) continue;
				const f3 d = f3_sub(pos[j], c);
				m3_add_outer(&Scur, d, d);
			}
			Scur = m3_scale(&Scur, invN);
			float J, C;
			m3 Sinv;
			if (!cluster_j_sinv(&Scur, S.det_rest[idx], &J, &C, &Sinv)) continue;
			const float gs = J * invN;
			float denom = 0.0f;
			{
				const f3 g = f3_mul(m3_mulv(&Sinv, f3_sub(pi, c)), gs);
				denom += (S.inv_mass[idx] * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
			}
			for (int k = 0; k < cnt; ++k) {
				const int j = S.vol_idx[off + k];
				if (j < 0 || j >= N) continue;
				const f3 g = f3_mul(m3_mulv(&Sinv, f3_sub(pos[j], c)), gs);
				denom += (S.inv_mass[j] * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
			}
			const float dt2 = fmaxf(dt * dt, 1e-8f);
			const float alphaT = P.vol_compliance / dt2;
			const float den = denom + alphaT;
			if (!(den > 1e-12f)) continue;
			const float lam = S.lam_vol[idx];
			const float dLam = (-C - alphaT * lam) / den;
			if (!isfinite(dLam)) continue;
			S.lam_vol[idx] = lam + dLam;
			const float coef = dLam * gs;
			/* leader then members, each clamped to 0.25 restLen (forward.cu:9150-9182) */
			for (int k = -1; k < cnt; ++k) {
				const int j = (k < 0) ? idx : S.vol_idx[off + k];
				if (j < 0 || j >= N) continue;
				const float wj = S.inv_mass[j] * ims;
				if (wj <= 0.0f) continue;
				const f3 pj = pos[j];
				const f3 g = m3_mulv(&Sinv, f3_sub(pj, c));
				f3 dp = mk3(g.x * wj * coef, g.y * wj * coef, g.z * wj * coef);
				if (!f3_finite(dp)) continue;
				const float rl = S.rest_len[j];
				if (rl > 1e-12f) {
					const float maxStep = 0.25f * rl;
					const float len = f3_len(dp);
					if (len > maxStep && len > 1e-20f) dp = f3_mul(dp, maxStep / len);
				}
				pos[j] = f3_add(pj, dp);
			}
		}
	}
}

/* shapeMatchRotationDouble (forward.cu:5991-6086) */
static int shape_rotation_double(const m3* A, m3* Rout)
{
	double a[3][3];
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c) a[r][c] = (double)A->m[c][r];
	double m[3][3];
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c) m[r][c] = a[0][r] * a[0][c] + a[1][r] * a[1][c] + a[2][r] * a[2][c];
	double v[3][3] = { { 1.0, 0.0, 0.0 }, { 0.0, 1.0, 0.0 }, { 0.0, 0.0, 1.0 } };
	const int Pp[3] = { 0, 0, 1 }, Qq[3] = { 1, 2, 2 };
	for (int iter = 0; iter < 50; ++iter) {
		int done = 1, p = 0, q = 1;
		double maxOff = -1.0;
		for (int k = 0; k < 3; ++k) {
			const double off = fabs(m[Pp[k]][Qq[k]]);
			if (off > 1e-12 * sqrt(fabs(m[Pp[k]][Pp[k]] * m[Qq[k]][Qq[k]])) + 1e-300) done = 0;
			if (off > maxOff) { maxOff = off; p = Pp[k]; q = Qq[k]; }
		}
		if (done) break;
		const double app = m[p][p], aqq = m[q][q], apq = m[p][q];
		const double phi = 0.5 * (aqq - app) / (apq + 1e-300);
		const double t = (phi >= 0.0) ? 1.0 / (phi + sqrt(1.0 + phi * phi)) : 1.0 / (phi - sqrt(1.0 + phi * phi));
		const double c = 1.0 / sqrt(1.0 + t * t);
		const double s = t * c;
		m[p][p] = app - t * apq;
		m[q][q] = aqq + t * apq;
		m[p][q] = m[q][p] = 0.0;
		for (int r = 0; r < 3; ++r) {
			if (r == p || r == q) continue;
			const double arp = m[r][p], arq = m[r][q];
			m[r][p] = m[p][r] = c * arp - s * arq;
			m[r][q] = m[q][r] = c * arq + s * arp;
		}
		for (int r = 0; r < 3; ++r) {
			const double vrp = v[r][p], vrq = v[r][q];
			v[r][p] = c * vrp - s * vrq;
			v[r][q] = s * vrp + c * vrq;
		}
	}
	double ev[3] = { m[0][0], m[1][1], m[2][2] };
	for (int i = 0; i < 2; ++i)
		for (int j = i + 1; j < 3; ++j)
			if (ev[i] > ev[j]) {
				const double te = ev[i]; ev[i] = ev[j]; ev[j] = te;
				for (int r = 0; r < 3; ++r) { const double tv = v[r][i]; v[r][i] = v[r][j]; v[r][j] = tv; }
			}
	double Sv[3], Sinv[3];
	for (int i = 0; i < 3; ++i) Sv[i] = sqrt(ev[i] > 0.0 ? ev[i] : 0.0);
	const double Smax = (Sv[2] > 1e-300) ? Sv[2] : 1e-300;
	for (int i = 0; i < 3; ++i) Sinv[i] = (Sv[i] > 1e-12 * Smax) ? 1.0 / Sv[i] : 0.0;
	double u[3][3];
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c) u[r][c] = (a[r][0] * v[0][c] + a[r][1] * v[1][c] + a[r][2] * v[2][c]) * Sinv[c];
	if (Sv[0] < 0.08 * Smax) {
		const double cx = u[1][1] * u[2][2] - u[2][1] * u[1][2];
		const double cy = u[2][1] * u[0][2] - u[0][1] * u[2][2];
		const double cz = u[0][1] * u[1][2] - u[1][1] * u[0][2];
		const double len = sqrt(cx * cx + cy * cy + cz * cz);
		if (!(len > 1e-7)) return 0;
		u[0][0] = cx / len; u[1][0] = cy / len; u[2][0] = cz / len;
	}
	double R[3][3];
	for (int pass = 0; pass < 2; ++pass) {
		for (int r = 0; r < 3; ++r)
			for (int c = 0; c < 3; ++c) R[r][c] = u[r][0] * v[c][0] + u[r][1] * v[c][1] + u[r][2] * v[c][2];
		const double det = R[0][0] * (R[1][1] * R[2][2] - R[1][2] * R[2][1])
			- R[0][1] * (R[1][0] * R[2][2] - R[1][2] * R[2][0])
			+ R[0][2] * (R[1][0] * R[2][1] - R[1][1] * R[2][0]);
		if (det >= 0.0 || pass == 1) break;
		for (int r = 0; r < 3; ++r) u[r][0] = -u[r][0];
	}
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c) {
			if (!isfinite(R[r][c])) return 0;
			Rout->m[c][r] = (float)R[r][c];
		}
	return 1;
}

static inline int m3_finite(const m3* M)
{
	for (int c = 0; c < 3; ++c)
		for (int r = 0; r < 3; ++r)
			if (!isfinite(M->m[c][r])) return 0;
	return 1;
}

/* float32 rotation path (forward.cu:6238-6319) */
static int shape_rotation_float(const m3* A, m3* Rout)
{
	m3 At = m3_transpose(A);
	m3 AtA = m3_mul(&At, A);
	f3 S2;
	m3 V;
	eig_glm(&AtA, &S2, &V);
	f3 Sv = mk3(sqrtf(fmaxf(0.0f, S2.x)), sqrtf(fmaxf(0.0f, S2.y)), sqrtf(fmaxf(0.0f, S2.z)));
	if (!f3_finite(Sv)) return 0;
	const float eps = 1e-7f;
	m3 Si = m3_zero();
	Si.m[0][0] = (Sv.x > eps) ? 1.0f / Sv.x : 0.0f;
	Si.m[1][1] = (Sv.y > eps) ? 1.0f / Sv.y : 0.0f;
	Si.m[2][2] = (Sv.z > eps) ? 1.0f / Sv.z : 0.0f;
	m3 AV = m3_mul(A, &V);
	m3 U = m3_mul(&AV, &Si);
	if (!m3_finite(&U)) return 0;
	if (Sv.x < 0.08f * fmaxf(Sv.z, 1e-7f)) {
		/* col0 = cross(U[1], U[2]) */
		const f3 u1 = mk3(U.m[1][0], U.m[1][1], U.m[1][2]);
		const f3 u2 = mk3(U.m[2][0], U.m[2][1], U.m[2][2]);
		const f3 cr = mk3(u1.y * u2.z - u2.y * u1.z, u1.z * u2.x - u2.z * u1.x, u1.x * u2.y - u2.x * u1.y);
		const float l = sqrtf(f3_dot(cr, cr));
		if (l > 1e-7f) { U.m[0][0] = cr.x / l; U.m[0][1] = cr.y / l; U.m[0][2] = cr.z / l; }
		else return 0;
	}
	m3 Vt = m3_transpose(&V);
	m3 R = m3_mul(&U, &Vt);
	if (!m3_finite(&R)) return 0;
	if (m3_det(&R) < 0.0f) {
		U.m[0][0] *= -1.0f; U.m[0][1] *= -1.0f; U.m[0][2] *= -1.0f;
		R = m3_mul(&U, &Vt);
		if (!m3_finite(&R)) return 0;
	}
	*Rout = R;
	return 1;
}

/* xpbdShapeMatchingKernel (forward.cu:6088-6383) + xpbdProjectTowardGoal (forward.cu:4972-4988) */
static void shape_matching(const f3* pin, f3* pout, float dt)
{
	const int N = S.n;
#pragma omp parallel for schedule(static) num_threads(nthreads())
	for (int idx = 0; idx < N; ++idx) {
		const f3 pi = pin[idx];
		const float wi = S.inv_mass[idx] * P.inv_mass_scale;
		if (wi <= 0.0f) { pout[idx] = pi; continue; }
		const int off = S.off[idx], cnt = S.cnt[idx];
		if (cnt < 4) { pout[idx] = pi; continue; }
		f3 comRest = S.pos_rest[idx];
		f3 comCurr = pi;
		float clusterCount = 1.0f;
		for (int k = 0; k < cnt; ++k) {
			const int nIdx = S.nbr[off + k];
			if (nIdx < 0 || nIdx >= N) continue;
			comRest = f3_add(comRest, S.pos_rest[nIdx]);
			comCurr = f3_add(comCurr, pin[nIdx]);
			clusterCount += 1.0f;
		}
		if (clusterCount < 2.0f) { pout[idx] = pi; continue; }
		const float invCluster = 1.0f / clusterCount;
		comRest = f3_mul(comRest, invCluster);
		comCurr = f3_mul(comCurr, invCluster);
		{
			f3 dirSum = mk3(0, 0, 0);
			float maxLen = 0.0f;
			for (int k = 0; k < cnt; ++k) {
				const int nIdx = S.nbr[off + k];
				if (nIdx < 0 || nIdx >= N) continue;
				const f3 q = f3_sub(S.pos_rest[nIdx], comRest);
				const float len = f3_len(q);
				if (len > 1e-7f) {
					dirSum = f3_add(dirSum, f3_mul(q, 1.0f / len));
					if (len > maxLen) maxLen = len;
				}
			}
			const float bias = f3_len(dirSum) / fmaxf((float)cnt, 1.0f);
			if (bias > 0.4f) { pout[idx] = pi; continue; }
		}
		m3 A = m3_zero();
		m3_add_outer(&A, f3_sub(pi, comCurr), f3_sub(S.pos_rest[idx], comRest));
		for (int k = 0; k < cnt; ++k) {
			const int nIdx = S.nbr[off + k];
			if (nIdx < 0 || nIdx >= N) continue;
			m3_add_outer(&A, f3_sub(pin[nIdx], comCurr), f3_sub(S.pos_rest[nIdx], comRest));
		}
		float a_norm_sq = 0.0f;
		for (int c = 0; c < 3; ++c)
			for (int r = 0; r < 3; ++r) a_norm_sq += A.m[c][r] * A.m[c][r];
		const float a_norm = sqrtf(a_norm_sq);
		if (!isfinite(a_norm) || a_norm < 1e-8f) { pout[idx] = pi; continue; }
		A = m3_divs(&A, a_norm);
		m3 R = m3_diag(1.0f);
		if (P.shape_robust) {
			if (!shape_rotation_double(&A, &R)) { pout[idx] = pi; continue; }
		}
		else if (!shape_rotation_float(&A, &R)) { pout[idx] = pi; continue; }
		const f3 qi = f3_sub(S.pos_rest[idx], comRest);
		const f3 rq = m3_mulv(&R, qi);
		const f3 goal = f3_add(comCurr, rq);
		const f3 gd = f3_sub(goal, pi);
		const float gd2 = f3_len2(gd);
		if (!isfinite(gd2) || gd2 < 1e-18f) { pout[idx] = pi; continue; }
		const float dt2 = fmaxf(dt * dt, 1e-8f);
		const float alphaTilde = P.shape_compliance / dt2;
		const float denom = wi + alphaTilde;
		if (denom < 1e-8f) { pout[idx] = pi; continue; }
		const float scale = P.shape_blend * (wi / denom);
		pout[idx] = f3_add(pi, f3_mul(f3_sub(goal, pi), scale));
	}
}

/* contactSupport (forward.cu:7387-7392): support distance sqrt(n^T M n) */
static inline float contact_support(const float* m, float nx, float ny, float nz)
{
	const float q = m[0] * nx * nx + m[3] * ny * ny + m[5] * nz * nz
		+ 2.0f * (m[1] * nx * ny + m[2] * nx * nz + m[4] * ny * nz);
	return sqrtf(fmaxf(q, 0.0f));
}

/* contactShapePackKernel (forward.cu:7358-7385) over n Gaussians */
static void contact_pack(const float* sc, const float* qt, const float* op, int n, float tau, float rcap)
{
	if (S.contact_n != n) {
		FREE(S.contact_M); FREE(S.contact_rmax); FREE(S.contact_rg);
		S.contact_M = malloc(sizeof(float) * 6 * n);
		S.contact_rmax = malloc(sizeof(float) * n);
		S.contact_rg = calloc(n, sizeof(float));
		S.contact_n = n;
	}
	for (int i = 0; i < n; ++i) {
		const float a = op[i];
		const float k = (a > tau && tau > 0.0f) ? sqrtf(2.0f * logf(a / tau)) : 0.0f;
		float e0 = k * sc[3 * i], e1 = k * sc[3 * i + 1], e2 = k * sc[3 * i + 2];
		if (rcap > 0.0f) { e0 = fminf(e0, rcap); e1 = fminf(e1, rcap); e2 = fminf(e2, rcap); }
		if (!(isfinite(e0) && isfinite(e1) && isfinite(e2))) { e0 = e1 = e2 = 0.0f; }
		float w = qt[4 * i], x = qt[4 * i + 1], y = qt[4 * i + 2], z = qt[4 * i + 3];
		const float qn = sqrtf(w * w + x * x + y * y + z * z);
		if (qn > 1e-20f) { w /= qn; x /= qn; y /= qn; z /= qn; } else { w = 1.0f; x = y = z = 0.0f; }
		const float r00 = 1 - 2 * (y * y + z * z), r01 = 2 * (x * y - w * z), r02 = 2 * (x * z + w * y);
		const float r10 = 2 * (x * y + w * z), r11 = 1 - 2 * (x * x + z * z), r12 = 2 * (y * z - w * x);
		const float r20 = 2 * (x * z - w * y), r21 = 2 * (y * z + w * x), r22 = 1 - 2 * (x * x + y * y);
		const float l0 = e0 * e0, l1 = e1 * e1, l2 = e2 * e2;
		float* m = &S.contact_M[6 * i];
		m[0] = r00 * r00 * l0 + r01 * r01 * l1 + r02 * r02 * l2;
		m[1] = r00 * r10 * l0 + r01 * r11 * l1 + r02 * r12 * l2;
		m[2] = r00 * r20 * l0 + r01 * r21 * l1 + r02 * r22 * l2;
		m[3] = r10 * r10 * l0 + r11 * r11 * l1 + r12 * r12 * l2;
		m[4] = r10 * r20 * l0 + r11 * r21 * l1 + r12 * r22 * l2;
		m[5] = r20 * r20 * l0 + r21 * r21 * l1 + r22 * r22 * l2;
		S.contact_rmax[i] = fmaxf(e0, fmaxf(e1, e2));
	}
}

/* kinColliderProjectKernel (forward.cu:7425-7518); cM / cRmax non-NULL: ellipsoid contacts */
static void colliders_project(f3* pos, int countHits, const float* cM, const float* cRmax)
{
	const int N = S.n, nc = P.kin_count;
	const float margin = P.kin_margin, mu = P.kin_friction;
	int hits[MAX_KIN] = { 0 };
	double acc[MAX_KIN * KIN_ACC];
	memset(acc, 0, sizeof(acc));
#pragma omp parallel num_threads(nthreads())
	{
		int lh[MAX_KIN] = { 0 };
		double la[MAX_KIN * KIN_ACC];
		memset(la, 0, sizeof(la));
#pragma omp for schedule(static)
		for (int idx = 0; idx < N; ++idx) {
			if (S.inv_mass[idx] <= 0.0f) continue;
			f3 p = pos[idx];
			int moved = 0;
			const float rmax = cRmax ? cRmax[idx] : 0.0f;
			const float reach = margin + rmax;
			for (int c = 0; c < nc; ++c) {
				const kin_t* C = &P.kin[c];
				const float dx = p.x - C->t[0], dy = p.y - C->t[1], dz = p.z - C->t[2];
				const float q0 = C->R[0] * dx + C->R[3] * dy + C->R[6] * dz;
				const float q1 = C->R[1] * dx + C->R[4] * dy + C->R[7] * dz;
				const float q2 = C->R[2] * dx + C->R[5] * dy + C->R[8] * dz;
				float n0 = 0.0f, n1 = 0.0f, n2 = 1.0f, dist;
				if (C->type == 1) {
					const float a0 = fabsf(q0) - C->h[0], a1 = fabsf(q1) - C->h[1], a2 = fabsf(q2) - C->h[2];
					if (a0 > 0.0f || a1 > 0.0f || a2 > 0.0f) {
						const float o0 = fmaxf(a0, 0.0f), o1 = fmaxf(a1, 0.0f), o2 = fmaxf(a2, 0.0f);
						dist = sqrtf(o0 * o0 + o1 * o1 + o2 * o2);
						if (dist >= reach) continue;
						const float inv = 1.0f / fmaxf(dist, 1e-20f);
						n0 = copysignf(o0 * inv, q0); n1 = copysignf(o1 * inv, q1); n2 = copysignf(o2 * inv, q2);
					}
					else {
						if (a0 >= a1 && a0 >= a2) { dist = a0; n0 = (q0 >= 0.0f) ? 1.0f : -1.0f; n2 = 0.0f; }
						else if (a1 >= a2) { dist = a1; n1 = (q1 >= 0.0f) ? 1.0f : -1.0f; n2 = 0.0f; }
						else { dist = a2; n2 = (q2 >= 0.0f) ? 1.0f : -1.0f; }
					}
				}
				else {
					float e2 = q2;
					if (C->type == 2) e2 = q2 - fminf(fmaxf(q2, -C->h[1]), C->h[1]);
					const float r = sqrtf(q0 * q0 + q1 * q1 + e2 * e2);
					dist = r - C->h[0];
					if (dist >= reach) continue;
					if (r > 1e-20f) { n0 = q0 / r; n1 = q1 / r; n2 = e2 / r; }
				}
				const float wx = C->R[0] * n0 + C->R[1] * n1 + C->R[2] * n2;
				const float wy = C->R[3] * n0 + C->R[4] * n1 + C->R[5] * n2;
				const float wz = C->R[6] * n0 + C->R[7] * n1 + C->R[8] * n2;
				if (cM && rmax > 0.0f) {
					dist -= contact_support(&cM[6 * idx], wx, wy, wz);
					if (dist >= margin) continue;
				}
				const float corr = margin - dist;
				const f3 pIn = p;
				p.x += wx * corr; p.y += wy * corr; p.z += wz * corr;
				f3 dp = mk3(wx * corr, wy * corr, wz * corr);
				if (mu > 0.0f) {
					const float ox = C->Rp[0] * q0 + C->Rp[1] * q1 + C->Rp[2] * q2 + C->tp[0];
					const float oy = C->Rp[3] * q0 + C->Rp[4] * q1 + C->Rp[5] * q2 + C->tp[1];
					const float oz = C->Rp[6] * q0 + C->Rp[7] * q1 + C->Rp[8] * q2 + C->tp[2];
					const f3 x0 = S.pos_curr[idx];
					const float rx = (p.x - x0.x) - (pIn.x - ox), ry = (p.y - x0.y) - (pIn.y - oy),
						rz = (p.z - x0.z) - (pIn.z - oz);
					const float rn = rx * wx + ry * wy + rz * wz;
					const float tx = rx - rn * wx, ty = ry - rn * wy, tz = rz - rn * wz;
					const float lt = sqrtf(tx * tx + ty * ty + tz * tz);
					if (lt > 1e-20f) {
						const float k = fminf(1.0f, mu * corr / lt);
						p.x -= k * tx; p.y -= k * ty; p.z -= k * tz;
						dp.x -= k * tx; dp.y -= k * ty; dp.z -= k * tz;
					}
				}
				moved = 1;
				const float w = sqrtf(dp.x * dp.x + dp.y * dp.y + dp.z * dp.z);
				double* a = &la[KIN_ACC * c];
				a[0] += dp.x; a[1] += dp.y; a[2] += dp.z;
				a[3] += w * p.x; a[4] += w * p.y; a[5] += w * p.z; a[6] += w;
				if (countHits) lh[c]++;
			}
			if (moved) pos[idx] = p;
		}
#pragma omp critical
		{
			for (int c = 0; c < nc; ++c) {
				hits[c] += lh[c];
				for (int k = 0; k < KIN_ACC; ++k) acc[KIN_ACC * c + k] += la[KIN_ACC * c + k];
			}
		}
	}
	for (int c = 0; c < nc; ++c) {
		if (countHits) P.kin_hits[c] += hits[c];
		for (int k = 0; k < KIN_ACC; ++k) P.kin_push[KIN_ACC * c + k] += (float)acc[KIN_ACC * c + k];
	}
}

/* groundProjectKernel (forward.cu:7405-7421); rg non-NULL: ellipsoid contacts */
static void ground_project(f3* pos, const float* rg)
{
	const f3 n = mk3(P.ground_n[0], P.ground_n[1], P.ground_n[2]);
	const float planeD = P.ground_h + P.ground_radius;
#pragma omp parallel for schedule(static) num_threads(nthreads())
	for (int i = 0; i < S.n; ++i) {
		if (S.inv_mass[i] <= 0.0f) continue;
		const f3 p = pos[i];
		const float c = n.x * p.x + n.y * p.y + n.z * p.z - planeD - (rg ? rg[i] : 0.0f);
		if (c < 0.0f) pos[i] = mk3(p.x - c * n.x, p.y - c * n.y, p.z - c * n.z);
	}
}

/* xpbdUpdateVelocityKernel (forward.cu:6623-6672) and ...GroundKernel (forward.cu:7528-7599) */
static void velocity_commit(const f3* pfinal, float dt, int groundOn, const float* rg)
{
	const float velDamping = P.vel_damping;
	const f3 n = mk3(P.ground_n[0], P.ground_n[1], P.ground_n[2]);
	const float planeD = P.ground_h + P.ground_radius, slop = P.ground_slop, friction = P.ground_fric,
		restitution = P.ground_rest, restingSpeed = 2.0f * P.ground_gravity * dt;
#pragma omp parallel for schedule(static) num_threads(nthreads())
	for (int idx = 0; idx < S.n; ++idx) {
		const f3 x = S.pos_curr[idx];
		const f3 p = pfinal[idx];
		const float w = S.inv_mass[idx];
		if (!groundOn) {
			if (w > 0.0f) {
				const f3 dx = f3_sub(p, x);
				const float dx2 = f3_len2(dx);
				if (!isfinite(dx2) || dx2 < 1e-18f) {
					S.vel[idx] = mk3(0, 0, 0);
					S.pos_curr[idx] = p;
					continue;
				}
				f3 vs = f3_mul(dx, 1.0f / fmaxf(dt, 1e-8f));
				const float damping = fminf(fmaxf(velDamping, 0.0f), 1.0f);
				const float retention = 1.0f - damping;
				vs = f3_mul(vs, retention);
				if (!f3_finite(vs) || f3_len2(vs) < 1e-16f) vs = mk3(0, 0, 0);
				S.vel[idx] = vs;
				S.pos_curr[idx] = p;
				continue;
			}
			S.vel[idx] = mk3(0, 0, 0);
			S.pos_curr[idx] = p;
			continue;
		}
		if (w <= 0.0f) { S.vel[idx] = mk3(0, 0, 0); S.pos_curr[idx] = p; continue; }
		const f3 vPre = S.vel[idx];
		const f3 dx = f3_sub(p, x);
		const float dx2 = f3_len2(dx);
		if (!isfinite(dx2)) { S.vel[idx] = mk3(0, 0, 0); S.pos_curr[idx] = p; continue; }
		f3 v = (dx2 < 1e-18f) ? mk3(0, 0, 0) : f3_mul(dx, 1.0f / fmaxf(dt, 1e-8f));
		const float gap = n.x * p.x + n.y * p.y + n.z * p.z - planeD - (rg ? rg[idx] : 0.0f);
		if (gap <= slop) {
			const float vn = n.x * v.x + n.y * v.y + n.z * v.z;
			const float vnPre = n.x * vPre.x + n.y * vPre.y + n.z * vPre.z;
			float vnNew = vn, jn = 0.0f;
			if (vnPre < 0.0f) {
				const float e = (-vnPre <= restingSpeed) ? 0.0f : restitution;
				vnNew = fmaxf(vn, -e * vnPre);
				jn = -(1.0f + e) * vnPre;
			}
			f3 vt = mk3(v.x - vn * n.x, v.y - vn * n.y, v.z - vn * n.z);
			const float vtLen = f3_len(vt);
			const float dvt = friction * jn;
			if (vtLen <= dvt || vtLen < 1e-12f) vt = mk3(0, 0, 0);
			else vt = f3_mul(vt, (vtLen - dvt) / vtLen);
			v = mk3(vt.x + vnNew * n.x, vt.y + vnNew * n.y, vt.z + vnNew * n.z);
		}
		const float damping = fminf(fmaxf(velDamping, 0.0f), 1.0f);
		v = f3_mul(v, 1.0f - damping);
		if (!f3_finite(v) || f3_len2(v) < 1e-16f) v = mk3(0, 0, 0);
		S.vel[idx] = v;
		S.pos_curr[idx] = p;
	}
}

/* ------------------------------------------------------------------------- */
/* self-collision (forward.cu:6984-7322, 11705-11849)                         */
/* ------------------------------------------------------------------------- */
static inline unsigned int sc_hash(int cx, int cy, int cz, unsigned int mask)
{
	return (((unsigned int)cx * 73856093u) ^ ((unsigned int)cy * 19349663u) ^ ((unsigned int)cz * 83492791u)) & mask;
}
static inline int sc_cell(float v, float invCell)
{
	return (int)floorf(fminf(fmaxf(v * invCell, -1.0e9f), 1.0e9f));
}

static int cmp_float(const void* a, const void* b)
{
	const float x = *(const float*)a, y = *(const float*)b;
	return (x < y) ? -1 : (x > y) ? 1 : 0;
}

/* selfColEnsureSpacing (forward.cu:11761-11792): median of per-node shortest graph edge */
static void sc_ensure_spacing(void)
{
	if (S.sc_spacing > 0.0f) return;
	if (S.m <= 0) return;
	float* mins = malloc(sizeof(float) * S.n);
	int nm = 0;
	for (int i = 0; i < S.n; ++i) {
		float m = FLT_MAX;
		for (int k = 0; k < S.cnt[i]; ++k) {
			const int e = S.off[i] + k;
			if (e < 0 || e >= S.m) continue;
			const float d = S.ndist[e];
			if (d > 0.0f && isfinite(d) && d < m) m = d;
		}
		if (m < FLT_MAX) mins[nm++] = m;
	}
	if (nm > 0) {
		qsort(mins, nm, sizeof(float), cmp_float);
		S.sc_spacing = mins[nm / 2];
	}
	free(mins);
}

/* objectEnsureComponents (forward.cu:11309-11374): graph components >= 50 are objects */
static int find_root(int* parent, int x)
{
	while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; }
	return x;
}
static void ensure_components(void)
{
	if (S.obj_id) return;
	const int N = S.n;
	int* parent = malloc(sizeof(int) * N);
	for (int i = 0; i < N; ++i) parent[i] = i;
	for (int i = 0; i < N; ++i)
		for (int k = 0; k < S.cnt[i]; ++k) {
			const int e = S.off[i] + k;
			if (e < 0 || e >= S.m) continue;
			const int j = S.nbr[e];
			if (j < 0 || j >= N) continue;
			const int ri = find_root(parent, i), rj = find_root(parent, j);
			if (ri != rj) parent[ri] = rj;
		}
	int* compSize = calloc(N, sizeof(int));
	for (int i = 0; i < N; ++i) ++compSize[find_root(parent, i)];
	int* rootId = malloc(sizeof(int) * N);
	for (int i = 0; i < N; ++i) rootId[i] = -1;
	S.obj_id = malloc(sizeof(int) * N);
	int K = 0;
	for (int i = 0; i < N; ++i) {
		const int r = find_root(parent, i);
		if (rootId[r] == -1) rootId[r] = (compSize[r] >= P.obj_min_component) ? K++ : -2;
		S.obj_id[i] = rootId[r] >= 0 ? rootId[r] : -1;
	}
	S.obj_k = K;
	free(parent); free(compSize); free(rootId);
}

static void sc_ensure_buffers(void)
{
	if (S.sc_table) return;
	const int N = S.n;
	int table = 1024;
	while (table < 2 * N) table <<= 1;
	int bits = 0;
	while ((1 << bits) < table) ++bits;
	S.sc_table = table;
	S.sc_bits = bits;
	S.sc_keys = malloc(sizeof(unsigned int) * N);
	S.sc_keys_sorted = malloc(sizeof(unsigned int) * N);
	S.sc_idx_sorted = malloc(sizeof(int) * N);
	S.sc_cell_start = malloc(sizeof(int) * table);
	S.sc_cell_end = malloc(sizeof(int) * table);
	S.sc_contact = malloc(sizeof(int) * (size_t)N * SC_MAX);
	S.sc_count = calloc(N, sizeof(int));
	S.sc_dp = calloc(N, sizeof(f3));
	S.sc_dp_cross = calloc(N, sizeof(f3));
}

/* selfColBuildKernel (forward.cu:7079-7180) for one particle */
static int sc_build_one(int i, const f3* X, const f3* Pp, float invCell, unsigned int mask, float search,
	float excludeR2, float crossExcludeR2, float fastRel, int* overflow)
{
	const f3 x = X[i], p = Pp[i];
	int cnt = 0;
	if (f3_finite(x) && f3_finite(p)) {
		const f3 q = S.pos_rest[i];
		const float dix = p.x - x.x, diy = p.y - x.y, diz = p.z - x.z;
		const int oi = S.obj_id[i];
		const float search2 = search * search;
		const int cx = sc_cell(x.x, invCell), cy = sc_cell(x.y, invCell), cz = sc_cell(x.z, invCell);
		int* out = S.sc_contact + (size_t)i * SC_MAX;
		unsigned int hs[27];
		float prio[SC_MAX];
		int tier[SC_MAX];
		int nh = 0;
		for (int oz = -1; oz <= 1; ++oz)
			for (int oy = -1; oy <= 1; ++oy)
				for (int ox = -1; ox <= 1; ++ox) {
					const unsigned int h = sc_hash(cx + ox, cy + oy, cz + oz, mask);
					int dup = 0;
					for (int m = 0; m < nh; ++m) if (hs[m] == h) { dup = 1; break; }
					if (dup) continue;
					hs[nh++] = h;
					const int s = S.sc_cell_start[h];
					if (s < 0) continue;
					const int e = S.sc_cell_end[h];
					for (int t = s; t < e; ++t) {
						const int j = S.sc_idx_sorted[t];
						if (j == i) continue;
						const int cross = (S.obj_id[j] != oi);
						if (!cross && !P.sc_within) continue;
						const f3 pj = Pp[j], qj = S.pos_rest[j];
						const float qx = q.x - qj.x, qy = q.y - qj.y, qz = q.z - qj.z;
						const float q2 = qx * qx + qy * qy + qz * qz;
						float pr;
						int code = j;
						if (cross) {
							const f3 xj = X[j];
							const float ex = x.x - xj.x, ey = x.y - xj.y, ez = x.z - xj.z;
							const float distX = sqrtf(ex * ex + ey * ey + ez * ez);
							const float rx = dix - (pj.x - xj.x), ry = diy - (pj.y - xj.y), rz = diz - (pj.z - xj.z);
							const float rel = sqrtf(rx * rx + ry * ry + rz * rz);
							if (!(distX < search + rel)) continue;
							if (!(q2 >= crossExcludeR2)) continue;
							pr = distX - rel;
							if (rel > fastRel) code = -(j + 1);
						}
						else {
							const float ex = p.x - pj.x, ey = p.y - pj.y, ez = p.z - pj.z;
							const float d2 = ex * ex + ey * ey + ez * ez;
							if (!(d2 < search2)) continue;
							if (!(q2 >= excludeR2)) continue;
							pr = sqrtf(d2);
						}
						const int tr = cross ? 0 : 1;
						if (cnt < SC_MAX) {
							out[cnt] = code; prio[cnt] = pr; tier[cnt] = tr; ++cnt;
						}
						else {
							int worst = 0;
							for (int m = 1; m < SC_MAX; ++m)
								if (tier[m] > tier[worst] || (tier[m] == tier[worst] && prio[m] > prio[worst])) worst = m;
							if (tr < tier[worst] || (tr == tier[worst] && pr < prio[worst])) {
								out[worst] = code; prio[worst] = pr; tier[worst] = tr;
							}
							++*overflow;
						}
					}
				}
	}
	S.sc_count[i] = cnt;
	return cnt;
}

/* selfColBuild (forward.cu:11796-11849); with `limited`, only the Gaussians near another
 * object's box take part (object mode, cross-object contacts only; forward.cu:11808-11816) */
static void sc_active_set(const f3* X, const f3* Pp, float search, float dc);
static void sc_build_active(const f3* X, const f3* Pp, int limited)
{
	const int N = S.n;
	sc_ensure_spacing();
	const float dc = P.sc_radius_scale * S.sc_spacing;
	if (!(dc > 0.0f)) { S.sc_contacts = 0; return; }
	sc_ensure_buffers();
	ensure_components();
	const float search = P.sc_search_scale * dc;
	const float excl = P.sc_exclude_scale * dc;
	const unsigned char* act = NULL;
	if (limited) {
		sc_active_set(X, Pp, search, dc);
		act = S.sc_act;
	}
	float maxDisp2 = 0.0f;
	for (int i = 0; i < N; ++i) {
		if (act && !act[i]) continue;
		const float dx = Pp[i].x - X[i].x, dy = Pp[i].y - X[i].y, dz = Pp[i].z - X[i].z;
		const float d2 = dx * dx + dy * dy + dz * dz;
		const float v = isfinite(d2) ? d2 : 0.0f;
		if (v > maxDisp2) maxDisp2 = v;
	}
	const float maxDisp = (isfinite(maxDisp2) && maxDisp2 > 0.0f) ? sqrtf(maxDisp2) : 0.0f;
	float reach = search + 2.0f * maxDisp;
	const float reachCap = search + 16.0f * dc;
	if (reach > reachCap) reach = reachCap;
	S.sc_reach = reach;
	const float invCell = 1.0f / reach;
	const unsigned int mask = (unsigned int)S.sc_table - 1u;
	const unsigned int sentinel = (unsigned int)S.sc_table;
	for (int i = 0; i < N; ++i) {
		const f3 p = X[i];
		if ((act && !act[i]) || !f3_finite(p)) { S.sc_keys[i] = sentinel; continue; }
		S.sc_keys[i] = sc_hash(sc_cell(p.x, invCell), sc_cell(p.y, invCell), sc_cell(p.z, invCell), mask);
	}
	/* stable counting sort by key = CUB's stable radix sort of (key, i) pairs */
	const int T = S.sc_table + 1;
	int* start = calloc((size_t)T + 1, sizeof(int));
	for (int i = 0; i < N; ++i) start[S.sc_keys[i] + 1]++;
	for (int k = 0; k < T; ++k) start[k + 1] += start[k];
	for (int i = 0; i < N; ++i) {
		const int pos = start[S.sc_keys[i]]++;
		S.sc_keys_sorted[pos] = S.sc_keys[i];
		S.sc_idx_sorted[pos] = i;
	}
	free(start);
	for (int k = 0; k < S.sc_table; ++k) S.sc_cell_start[k] = -1;
	for (int i = 0; i < N; ++i) {
		const unsigned int k = S.sc_keys_sorted[i];
		if (k > mask) continue;
		if (i == 0 || S.sc_keys_sorted[i - 1] != k) S.sc_cell_start[k] = i;
		if (i == N - 1 || S.sc_keys_sorted[i + 1] != k) S.sc_cell_end[k] = i + 1;
	}
	long long total = 0, over = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total, over) num_threads(nthreads())
	for (int i = 0; i < N; ++i) {
		int ov = 0;
		if (act && !act[i]) { S.sc_count[i] = 0; continue; }
		total += sc_build_one(i, X, Pp, invCell, mask, search, excl * excl, dc * dc, P.sc_fast_rel * dc, &ov);
		over += ov;
	}
	S.sc_contacts = (int)total;
	S.sc_overflow = (int)over;
	int na = N;
	if (act) { na = 0; for (int i = 0; i < N; ++i) na += act[i] ? 1 : 0; }
	S.sc_active = na;
}

static void sc_build(const f3* X, const f3* Pp) { sc_build_active(X, Pp, 0); }

/* selfColStartNormal (forward.cu:7183-7197) */
static inline int sc_start_normal(f3 xi, f3 xj, f3 qi, f3 qj, float* nx, float* ny, float* nz)
{
	*nx = xi.x - xj.x; *ny = xi.y - xj.y; *nz = xi.z - xj.z;
	float l2 = *nx * *nx + *ny * *ny + *nz * *nz;
	if (!(l2 > 1e-24f)) {
		*nx = qi.x - qj.x; *ny = qi.y - qj.y; *nz = qi.z - qj.z;
		l2 = *nx * *nx + *ny * *ny + *nz * *nz;
		if (!(l2 > 1e-24f)) return 0;
	}
	const float inv = 1.0f / sqrtf(l2);
	*nx *= inv; *ny *= inv; *nz *= inv;
	return 1;
}

/* selfColSolveKernel + selfColApplyKernel (forward.cu:7205-7322) */
static void sc_solve_apply(f3* pos, f3* accum)
{
	const int N = S.n;
	const float dc = P.sc_radius_scale * S.sc_spacing;
	const float ims = P.inv_mass_scale;
#pragma omp parallel for schedule(static) num_threads(nthreads())
	for (int i = 0; i < N; ++i) {
		const int cnt = S.sc_count[i];
		if (cnt <= 0) continue;
		const float wi = S.inv_mass[i] * ims;
		float ax = 0, ay = 0, az = 0;
		int act = 0;
		float cpx = 0, cpy = 0, cpz = 0, sx = 0, sy = 0, sz = 0, wFast = 0;
		int nFast = 0;
		const int* list = S.sc_contact + (size_t)i * SC_MAX;
		if (wi > 0.0f) {
			const f3 pi = pos[i], xi = S.pos_curr[i], qi = S.pos_rest[i];
			const float dc2 = dc * dc;
			for (int k = 0; k < cnt; ++k) {
				const int code = list[k];
				if (code < 0) {
					const int j = -code - 1;
					float nx, ny, nz;
					if (!sc_start_normal(xi, S.pos_curr[j], qi, S.pos_rest[j], &nx, &ny, &nz)) continue;
					const f3 pj = pos[j];
					const float proj = (pi.x - pj.x) * nx + (pi.y - pj.y) * ny + (pi.z - pj.z) * nz;
					if (!(proj < dc)) continue;
					const float pen = dc - proj;
					sx += nx * pen; sy += ny * pen; sz += nz * pen;
					const float wj = S.inv_mass[j] * ims;
					wFast += wi / (wi + wj);
					++nFast;
					continue;
				}
				const int j = code;
				const f3 pj = pos[j];
				const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
				const float d2 = dx * dx + dy * dy + dz * dz;
				if (!(d2 < dc2)) continue;
				const float wj = S.inv_mass[j] * ims;
				const float wr = wi / (wi + wj);
				if (d2 < 1e-24f) {
					const f3 qj = S.pos_rest[j];
					const float rx = qi.x - qj.x, ry = qi.y - qj.y, rz = qi.z - qj.z;
					const float r2 = rx * rx + ry * ry + rz * rz;
					if (!(r2 > 1e-24f)) continue;
					const float s = dc * wr / sqrtf(r2);
					ax += rx * s; ay += ry * s; az += rz * s;
					++act;
					continue;
				}
				const float d = sqrtf(d2);
				const float s = (dc - d) / d * wr;
				ax += dx * s; ay += dy * s; az += dz * s;
				++act;
			}
		}
		f3 out = (act > 0) ? mk3(ax / act, ay / act, az / act) : mk3(0, 0, 0);
		if (nFast > 0) {
			const float sl = sqrtf(sx * sx + sy * sy + sz * sz);
			if (sl > 1e-20f) {
				const float bx = sx / sl, by = sy / sl, bz = sz / sl;
				const f3 pi = pos[i], xi = S.pos_curr[i], qi = S.pos_rest[i];
				float delta = 0.0f;
				for (int k = 0; k < cnt; ++k) {
					const int code = list[k];
					if (code >= 0) continue;
					const int j = -code - 1;
					float nx, ny, nz;
					if (!sc_start_normal(xi, S.pos_curr[j], qi, S.pos_rest[j], &nx, &ny, &nz)) continue;
					const f3 pj = pos[j];
					const float ddx = pi.x - pj.x, ddy = pi.y - pj.y, ddz = pi.z - pj.z;
					if (!(ddx * nx + ddy * ny + ddz * nz < dc)) continue;
					const float pen = dc - (ddx * bx + ddy * by + ddz * bz);
					if (pen > delta) delta = pen;
				}
				if (delta > 0.0f) {
					const float sc = delta * (wFast / (float)nFast);
					cpx = bx * sc; cpy = by * sc; cpz = bz * sc;
					out = mk3(out.x + cpx, out.y + cpy, out.z + cpz);
				}
			}
		}
		S.sc_dp[i] = out;
		S.sc_dp_cross[i] = mk3(cpx, cpy, cpz);
	}
#pragma omp parallel for schedule(static) num_threads(nthreads())
	for (int i = 0; i < N; ++i) {
		if (S.sc_count[i] <= 0) continue;
		pos[i] = f3_add(pos[i], S.sc_dp[i]);
		if (accum) accum[i] = f3_add(accum[i], S.sc_dp_cross[i]);
	}
}

/* computeVolumeJKernel (forward.cu:9428-9476) + host stats (forward.cu:12658-12706) */
static void volume_j_stats(void)
{
	const int N = S.n;
	double wSum = 0.0, wJ = 0.0, wJ2 = 0.0;
	for (int idx = 0; idx < N; ++idx) {
		if (S.mat_type[idx] != 0) continue;
		float J = 1.0f;
		const int off = S.vol_off[idx], cnt = S.vol_cnt[idx];
		f3 c = S.pos_curr[idx];
		int used = 0;
		for (int k = 0; k < cnt; ++k) {
			const int j = S.vol_idx[off + k];
			if (j < 0 || j >= N) continue;
			c = f3_add(c, S.pos_curr[j]);
			++used;
		}
		if (used >= 3) {
			const float invN = 1.0f / (float)(used + 1);
			c = f3_mul(c, invN);
			m3 Sm = m3_zero();
			{
				const f3 d = f3_sub(S.pos_curr[idx], c);
				m3_add_outer(&Sm, d, d);
			}
			for (int k = 0; k < cnt; ++k) {
				const int j = S.vol_idx[off + k];
				if (j < 0 || j >= N) continue;
				const f3 d = f3_sub(S.pos_curr[j], c);
				m3_add_outer(&Sm, d, d);
			}
			Sm = m3_scale(&Sm, invN);
			float sCur, detHat;
			if (sigma_scale_det(&Sm, &sCur, &detHat)) {
				const float detCur = sCur * sCur * sCur * detHat;
				const float dRest = S.det_rest[idx];
				if (dRest >= 1e-30f) {
					const float Jc = sqrtf(detCur / dRest);
					if (isfinite(Jc) && Jc > 0.0f) J = Jc;
				}
			}
		}
		const double v = (double)S.v_rest[idx];
		if (v > 0.0 && isfinite(v)) { wSum += v; wJ += v * J; wJ2 += v * (double)J * J; }
	}
	if (wSum > 0.0) {
		const double m = wJ / wSum;
		S.jvw_mean = (float)m;
		S.jvw_std = (float)sqrt(fmax(0.0, wJ2 / wSum - m * m));
	}
}

/* ------------------------------------------------------------------------- */
/* object mode: rigid shape keeping per object after predict                  */
/* (forward.cu:12141-12166; device path 6801-6958, 11671-11702)               */
/* ------------------------------------------------------------------------- */
#define OBJ_MAX_K 64   /* OBJ_GPU_MAX_K (forward.cu:192) */
static int g_obj_gpu = 1;  /* g_objShapeGPU (forward.cu:193) */

/* objectEnsureRestCache (forward.cu:11376-11440) */
static void obj_ensure_cache(void)
{
	if (S.obj_cache) return;
	ensure_components();
	const int N = S.n, K = S.obj_k;
	double* sum = calloc(3 * (size_t)(K > 0 ? K : 1), sizeof(double));
	S.obj_count = calloc(K > 0 ? K : 1, sizeof(int));
	for (int i = 0; i < N; ++i) {
		const int id = S.obj_id[i];
		if (id < 0) continue;
		sum[3 * id] += S.pos_rest[i].x; sum[3 * id + 1] += S.pos_rest[i].y; sum[3 * id + 2] += S.pos_rest[i].z;
		S.obj_count[id]++;
	}
	S.obj_c0 = malloc(sizeof(float) * 3 * (K > 0 ? K : 1));
	S.obj_shift = malloc(sizeof(double) * 3 * (K > 0 ? K : 1));
	for (int k = 0; k < K; ++k)
		for (int a = 0; a < 3; ++a) {
			const int c = S.obj_count[k] > 0 ? S.obj_count[k] : 1;
			S.obj_c0[3 * k + a] = (float)(sum[3 * k + a] / c);
			S.obj_shift[3 * k + a] = (double)S.obj_c0[3 * k + a];
		}
	free(sum);
	S.obj_q = calloc(3 * (size_t)N, sizeof(double));
	S.obj_sumq = calloc(3 * (size_t)(K > 0 ? K : 1), sizeof(double));
	for (int i = 0; i < N; ++i) {
		const int id = S.obj_id[i];
		if (id < 0) continue;
		S.obj_q[3 * i] = (double)(S.pos_rest[i].x - S.obj_c0[3 * id]);
		S.obj_q[3 * i + 1] = (double)(S.pos_rest[i].y - S.obj_c0[3 * id + 1]);
		S.obj_q[3 * i + 2] = (double)(S.pos_rest[i].z - S.obj_c0[3 * id + 2]);
		for (int a = 0; a < 3; ++a) S.obj_sumq[3 * id + a] += S.obj_q[3 * i + a];
	}
	S.obj_params = calloc(16 * (size_t)(K > 0 ? K : 1), sizeof(float));
	S.obj_disp = calloc(K > 0 ? K : 1, sizeof(float));
	S.obj_boxes = calloc(6 * (size_t)(K > 0 ? K : 1), sizeof(float));
	S.obj_accum = calloc(N, sizeof(f3));
	S.sc_act = calloc(N, 1);
	if (!S.obj_w) {
		S.obj_w = malloc(sizeof(float) * N);
		for (int i = 0; i < N; ++i) S.obj_w[i] = 1.0f;
	}
	S.obj_shift_valid = 0;
	S.obj_cache = 1;
}

static int object_on(void) { return P.obj_shape > 0.0f && S.obj_k > 0; }
static int object_on_ensure(void)
{
	if (!(P.obj_shape > 0.0f) || Q.active) return 0;   /* objShape (forward.cu:12141) */
	obj_ensure_cache();
	return object_on();
}

/* objectShapeAccumKernel + objectShapeSolveKernel + objectBoxesKernel +
 * objectShapeMatchKernel, in that order, on the predicted positions */
static void object_step(f3* pos)
{
	const int N = S.n, K = S.obj_k;
	const int wOn = S.att_active && g_obj_gpu && K <= OBJ_MAX_K;
	const int stride = wOn ? 16 : 12;
	double* sums = calloc((size_t)K * 16, sizeof(double));
	for (int i = 0; i < N; ++i) {
		const int id = S.obj_id[i];
		if (id < 0) continue;
		const f3 p = pos[i];
		const double dx = (double)p.x - S.obj_shift[3 * id], dy = (double)p.y - S.obj_shift[3 * id + 1],
			dz = (double)p.z - S.obj_shift[3 * id + 2];
		const double qx = S.obj_q[3 * i], qy = S.obj_q[3 * i + 1], qz = S.obj_q[3 * i + 2];
		double v[16] = { dx, dy, dz, dx * qx, dx * qy, dx * qz, dy * qx, dy * qy, dy * qz, dz * qx, dz * qy, dz * qz,
			0, 0, 0, 0 };
		if (wOn) {
			const double w = (double)S.obj_w[i];
			for (int k = 0; k < 12; ++k) v[k] *= w;
			v[12] = w; v[13] = w * qx; v[14] = w * qy; v[15] = w * qz;
		}
		for (int k = 0; k < stride; ++k) sums[16 * id + k] += v[k];
	}
	for (int k = 0; k < K; ++k) {
		const double* Sk = &sums[16 * k];
		float* Pk = &S.obj_params[16 * k];
		const int n = S.obj_count[k];
		if (n < 4) { Pk[15] = 0.0f; S.obj_disp[k] = 0.0f; continue; }
		const double W = wOn ? Sk[12] : (double)n;
		if (!(W > 0.0)) { Pk[15] = 0.0f; S.obj_disp[k] = 0.0f; continue; }
		const double inv = 1.0 / W;
		const double dc[3] = { Sk[0] * inv, Sk[1] * inv, Sk[2] * inv };
		const double* sq = wOn ? &Sk[13] : &S.obj_sumq[3 * k];
		double a[9];
		for (int r = 0; r < 3; ++r)
			for (int c = 0; c < 3; ++c) a[3 * r + c] = Sk[3 + 3 * r + c] - dc[r] * sq[c];
		double now[3];
		for (int t = 0; t < 3; ++t) { now[t] = S.obj_shift[3 * k + t] + dc[t]; S.obj_shift[3 * k + t] = now[t]; }
		S.obj_disp[k] = (float)sqrt(dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2]);
		double fn = 0.0;
		for (int t = 0; t < 9; ++t) fn += a[t] * a[t];
		fn = sqrt(fn);
		if (!(fn > 1e-300) || !isfinite(fn)) { Pk[15] = 0.0f; continue; }
		m3 A, R;
		for (int r = 0; r < 3; ++r)
			for (int c = 0; c < 3; ++c) A.m[c][r] = (float)(a[3 * r + c] / fn);
		if (!shape_rotation_double(&A, &R)) { Pk[15] = 0.0f; continue; }
		for (int t = 0; t < 3; ++t) {
			Pk[t] = wOn ? (float)((double)S.obj_c0[3 * k + t] + Sk[13 + t] * inv) : S.obj_c0[3 * k + t];
			Pk[3 + t] = (float)now[t];
			for (int cc = 0; cc < 3; ++cc) Pk[6 + 3 * t + cc] = R.m[cc][t];
		}
		Pk[15] = 1.0f;
	}
	free(sums);
	if (P.sc_enabled && K <= OBJ_MAX_K) {
		for (int k = 0; k < K; ++k)
			for (int a = 0; a < 6; ++a) S.obj_boxes[6 * k + a] = (a < 3) ? FLT_MAX : -FLT_MAX;
		for (int i = 0; i < N; ++i) {
			const int id = S.obj_id[i];
			const f3 p = pos[i];
			if (id < 0 || !f3_finite(p)) continue;
			float* b = &S.obj_boxes[6 * id];
			b[0] = fminf(b[0], p.x); b[1] = fminf(b[1], p.y); b[2] = fminf(b[2], p.z);
			b[3] = fmaxf(b[3], p.x); b[4] = fmaxf(b[4], p.y); b[5] = fmaxf(b[5], p.z);
		}
	}
	const float s = P.obj_shape;
	for (int i = 0; i < N; ++i) {
		const int id = S.obj_id[i];
		if (id < 0 || S.inv_mass[i] <= 0.0f) continue;
		const float* Pk = &S.obj_params[16 * id];
		if (Pk[15] == 0.0f) continue;
		const f3 r = S.pos_rest[i], p = pos[i];
		const float qx = r.x - Pk[0], qy = r.y - Pk[1], qz = r.z - Pk[2];
		const float gx = Pk[3] + Pk[6] * qx + Pk[7] * qy + Pk[8] * qz;
		const float gy = Pk[4] + Pk[9] * qx + Pk[10] * qy + Pk[11] * qz;
		const float gz = Pk[5] + Pk[12] * qx + Pk[13] * qy + Pk[14] * qz;
		pos[i] = mk3(p.x + s * (gx - p.x), p.y + s * (gy - p.y), p.z + s * (gz - p.z));
	}
}

/* selfColActiveKernel (forward.cu:6998-7029) */
static void sc_active_set(const f3* X, const f3* Pp, float search, float dc)
{
	const int K = S.obj_k;
	float md = 0.0f;
	for (int k = 0; k < K; ++k) md = fmaxf(md, S.obj_disp[k]);
	const float inflate = search + 2.0f * md + 2.0f * dc;
	for (int i = 0; i < S.n; ++i) {
		const int id = S.obj_id[i];
		unsigned char a = 0;
		if (id < 0) a = 1;
		else {
			const f3 p = Pp[i], x = X[i];
			for (int k = 0; k < K; ++k) {
				if (k == id) continue;
				const float* b = &S.obj_boxes[6 * k];
				const float lx = b[0] - inflate, ly = b[1] - inflate, lz = b[2] - inflate;
				const float hx = b[3] + inflate, hy = b[4] + inflate, hz = b[5] + inflate;
				const int inP = p.x >= lx && p.x <= hx && p.y >= ly && p.y <= hy && p.z >= lz && p.z <= hz;
				const int inX = x.x >= lx && x.x <= hx && x.y >= ly && x.y <= hy && x.z >= lz && x.z <= hz;
				if (inP || inX) { a = 1; break; }
			}
		}
		S.sc_act[i] = a;
	}
}

/* objectContactPush (forward.cu:11858-11890) and the ground re-projection after it
 * (forward.cu:12587-12597) */
static void object_contact_push(f3* pos, const float* rg)
{
	const int N = S.n, K = S.obj_k;
	float* sums = calloc((size_t)K * 4, sizeof(float));
	for (int i = 0; i < N; ++i) {
		const int id = S.obj_id[i];
		if (id < 0) continue;
		const f3 a = S.obj_accum[i];
		if (!(a.x * a.x + a.y * a.y + a.z * a.z > 1e-30f)) continue;
		float* Sm = &sums[4 * id];
		Sm[0] += a.x; Sm[1] += a.y; Sm[2] += a.z; Sm[3] += 1.0f;
	}
	float* T = calloc((size_t)K * 4, sizeof(float));
	for (int k = 0; k < K; ++k) {
		const float n = sums[4 * k + 3];
		if (!(n > 0.0f)) continue;
		const float sc = P.obj_shape / n;
		const float tx = sums[4 * k] * sc, ty = sums[4 * k + 1] * sc, tz = sums[4 * k + 2] * sc;
		if (!isfinite(tx) || !isfinite(ty) || !isfinite(tz)) continue;
		T[4 * k] = tx; T[4 * k + 1] = ty; T[4 * k + 2] = tz; T[4 * k + 3] = 1.0f;
	}
	for (int i = 0; i < N; ++i) {
		const int id = S.obj_id[i];
		if (id < 0 || S.inv_mass[i] <= 0.0f) continue;
		const float* Tk = &T[4 * id];
		if (Tk[3] == 0.0f) continue;
		const f3 a = S.obj_accum[i];
		if (a.x * a.x + a.y * a.y + a.z * a.z > 1e-30f) continue;
		pos[i] = mk3(pos[i].x + Tk[0], pos[i].y + Tk[1], pos[i].z + Tk[2]);
	}
	free(sums);
	free(T);
	if (P.ground_on) ground_project(pos, rg);
}

/* ------------------------------------------------------------------------- */
/* one step: runXPBDSimulation (forward.cu:12038-12751) via stepPhysicsOnly  */
/* (forward.cu:13253-13264)                                                   */
/* ------------------------------------------------------------------------- */
/* the press ramp with its checkpoint dwells, once per step (forward.cu:12095-12111) */
static void press_advance(void)
{
	static const float ckpt[4] = { 0.25f, 0.50f, 0.75f, 1.00f };
	if (!Q.active) return;
	if (Q.autolog && Q.dwell > 0) {
		if (--Q.dwell == 0) ++Q.ckpt;
		return;
	}
	Q.cur = fminf(Q.cur + Q.ramp * P.dt, Q.max);
	if (Q.autolog && Q.ckpt < 4) {
		const float target = ckpt[Q.ckpt] * Q.max;
		if (Q.cur >= target) { Q.cur = target; Q.dwell = 90; }
	}
}

/* squashPressProjectKernel (forward.cu:9411-9424) */
static void press_project(f3* pos)
{
	const float lo = Q.lo + (Q.from_lo ? Q.cur : 0.0f), hi = Q.hi - (Q.from_lo ? 0.0f : Q.cur);
	const int ax = Q.axis;
#pragma omp parallel for schedule(static) num_threads(nthreads())
	for (int i = 0; i < S.n; ++i) {
		if (S.inv_mass[i] <= 0.0f) continue;
		f3 p = pos[i];
		const float v = ax == 0 ? p.x : (ax == 1 ? p.y : p.z);
		if (!(v < lo) && !(v > hi)) continue;
		const float t = (v < lo) ? lo : hi;
		if (ax == 0) p.x = t; else if (ax == 1) p.y = t; else p.z = t;
		pos[i] = p;
	}
}

static void run_step(void)
{
	const int N = S.n;
	const float dt = P.dt;
	press_advance();
	const f3 gravity = (P.ground_gravity > 0.0f && !Q.active)
		? mk3(-P.ground_gravity * P.ground_n[0], -P.ground_gravity * P.ground_n[1], -P.ground_gravity * P.ground_n[2])
		: mk3(0, 0, 0);
	if (P.use_distance && S.m > 0) {
		memset(S.lam_a, 0, sizeof(float) * S.m);
		memset(S.lam_b, 0, sizeof(float) * S.m);
	}
	if (P.use_volume) memset(S.lam_vol, 0, sizeof(float) * N);
	const int distGS = P.use_distance && P.dist_gs && S.gs_nedges > 0;
	const int volGS = P.use_volume && P.vol_gs && S.vol_gs_ncolors > 0;
	if (distGS) memset(S.gs_lam, 0, sizeof(float) * S.gs_nedges);
	const int groundOn = P.ground_on && !Q.active;   /* forward.cu:12140 */
	const int scOn = P.sc_enabled && !Q.active;       /* forward.cu:12179 */
	/* ellipsoid contacts (forward.cu:12222-12228): the ground radius once per step */
	const int contactOn = (S.contact_col || S.contact_ground) && S.contact_M && S.contact_n == N;
	const float* cRg = NULL;
	if (contactOn && S.contact_ground && groundOn) {
		for (int i = 0; i < N; ++i)
			S.contact_rg[i] = contact_support(&S.contact_M[6 * i], P.ground_n[0], P.ground_n[1], P.ground_n[2]);
		cRg = S.contact_rg;
	}
	const float* cM = (contactOn && S.contact_col) ? S.contact_M : NULL;
	const float* cRmax = (contactOn && S.contact_col) ? S.contact_rmax : NULL;
	predict(gravity, dt);
	const int objOn = object_on_ensure();
	int limited = 0;
	if (objOn) {
		limited = P.sc_enabled && !P.sc_within && S.obj_shift_valid && S.obj_k >= 1 && S.obj_k <= OBJ_MAX_K;
		object_step(S.pos_next);
		S.obj_shift_valid = 1;
	}
	int scContacts = 0;
	if (scOn) {
		sc_build_active(S.pos_curr, S.pos_next, limited);
		scContacts = S.sc_contacts;
		if (objOn && scContacts > 0) memset(S.obj_accum, 0, sizeof(f3) * N);
	}
	else S.sc_contacts = 0;
	if (P.kin_count > 0) {
		memset(P.kin_hits, 0, sizeof(P.kin_hits));
		memset(P.kin_push, 0, sizeof(P.kin_push));
	}
	f3* pin = S.pos_next;
	f3* pout = S.pos_tmp;
	float* lin = S.lam_a;
	float* lout = S.lam_b;
	const int warp = vol_use_warp();
	for (int it = 0; it < P.iters; ++it) {
		if (distGS) distance_gs(pin, dt);
		else if (P.use_distance) {
			distance_jacobi(pin, pout, lin, lout, dt);
			f3* t = pin; pin = pout; pout = t;
			float* tl = lin; lin = lout; lout = tl;
		}
		if (P.use_volume) {
			if (volGS) volume_gs(pin, dt);
			else {
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads())
				for (int i = 0; i < N; ++i) {
					if (warp) cluster_solve_warp(i, pin, dt);
					else cluster_solve_thread(i, pin, dt);
				}
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads())
				for (int i = 0; i < N; ++i) pout[i] = warp ? gather_warp(i, pin) : gather_thread(i, pin);
				f3* t = pin; pin = pout; pout = t;
			}
		}
		if (P.use_shape) {
			shape_matching(pin, pout, dt);
			f3* t = pin; pin = pout; pout = t;
		}
		if (Q.active) press_project(pin);
		if (scOn && scContacts > 0) sc_solve_apply(pin, objOn ? S.obj_accum : NULL);
		if (P.kin_count > 0) colliders_project(pin, it == P.iters - 1, cM, cRmax);
		if (groundOn) ground_project(pin, cRg);
	}
	if (objOn && scOn && scContacts > 0) object_contact_push(pin, cRg);
	velocity_commit(pin, dt, groundOn, cRg);
	if (P.jstats && P.use_volume >= 0) volume_j_stats();
}

/* ------------------------------------------------------------------------- */
/* C ABI (capi:66-310)                                                        */
/* ------------------------------------------------------------------------- */
EXPORT const char* xpbd_last_error(void) { return S.err; }

EXPORT int xpbd_create(int n, const float* pos, const float* scales, const float* rots, const float* opacity, int e,
	const int* edges, const float* rest, const float* stiff)
{
	free_all();
	if (n <= 0 || !pos || !scales || !rots || !opacity || e < 0 || (e > 0 && (!edges || !rest || !stiff)))
		return fail("xpbd_create: invalid arguments");
	S.n = n;
	S.n_edges = e;
	S.pos_in = malloc(sizeof(float) * 3 * n); memcpy(S.pos_in, pos, sizeof(float) * 3 * n);
	S.scales = malloc(sizeof(float) * 3 * n); memcpy(S.scales, scales, sizeof(float) * 3 * n);
	S.rots = malloc(sizeof(float) * 4 * n); memcpy(S.rots, rots, sizeof(float) * 4 * n);
	S.opacity = malloc(sizeof(float) * n); memcpy(S.opacity, opacity, sizeof(float) * n);
	S.edges = malloc(sizeof(int) * 2 * (e > 0 ? e : 1));
	S.edge_rest = malloc(sizeof(float) * (e > 0 ? e : 1));
	S.edge_stiff = malloc(sizeof(float) * (e > 0 ? e : 1));
	if (e > 0) {
		memcpy(S.edges, edges, sizeof(int) * 2 * e);
		memcpy(S.edge_rest, rest, sizeof(float) * e);
		memcpy(S.edge_stiff, stiff, sizeof(float) * e);
	}
	S.created = 1;
	S.built = 0;
	return 0;
}

EXPORT void xpbd_destroy(void)
{
	P.kin_count = 0;
	free_all();
}

EXPORT int xpbd_count(void) { return S.n; }

/* setXPBDParams (forward.cu:4896-4922) */
EXPORT void xpbd_set_solver(int iters, float dt, float underRelax, float velDamping, float stiffnessScale,
	float invMassScale, float distCompliance, float shapeCompliance, float shapeBlend, float angleCompliance,
	float angleBlend)
{
	P.iters = iters < 1 ? 1 : iters;
	P.dt = fmaxf(1e-5f, dt);
	P.under_relax = fmaxf(0.0f, underRelax);
	P.vel_damping = fmaxf(0.0f, velDamping);
	P.stiffness_scale = fmaxf(0.0f, stiffnessScale);
	P.inv_mass_scale = fmaxf(0.0f, invMassScale);
	P.dist_compliance = fmaxf(0.0f, distCompliance);
	P.shape_compliance = fmaxf(0.0f, shapeCompliance);
	P.shape_blend = fminf(fmaxf(0.0f, shapeBlend), 1.0f);
	P.angle_compliance = fmaxf(0.0f, angleCompliance);
	P.angle_blend = fminf(fmaxf(0.0f, angleBlend), 1.0f);
}

EXPORT void xpbd_set_constraints(int distance, int shape, int angle, int volume)
{
	P.use_distance = distance != 0;
	P.use_shape = shape != 0;
	P.use_angle = angle != 0;
	P.use_volume = volume != 0;
}

/* setVolumeParams / setVolumeRingK / setVolumeLeaderParams (forward.cu:3849, 3934-3966) */
EXPORT void xpbd_set_volume(float compliance, int ringK, int maxMembers, int leaderMinHop)
{
	P.vol_compliance = compliance;
	ringK = ringK < 1 ? 1 : (ringK > 8 ? 8 : ringK);
	maxMembers = maxMembers < 8 ? 8 : (maxMembers > 8192 ? 8192 : maxMembers);
	P.ring_k = ringK;
	P.max_members = maxMembers;
	P.topo_dirty = 1;
	leaderMinHop = leaderMinHop < 1 ? 1 : (leaderMinHop > 8 ? 8 : leaderMinHop);
	if (!(P.leader_min_hop == leaderMinHop && P.member_select == 1)) {
		P.leader_min_hop = leaderMinHop;
		P.member_select = 1;
		P.topo_dirty = 1;
	}
}

/* setGroundParams (forward.cu:4430-4446) */
EXPORT void xpbd_set_ground(int enabled, float ux, float uy, float uz, float height, float friction,
	float restitution, float contactRadius, float contactSlop, float gravity)
{
	float nx = ux, ny = uy, nz = uz;
	const float len = sqrtf(nx * nx + ny * ny + nz * nz);
	if (!(len > 1e-8f) || !isfinite(len)) { nx = 0.0f; ny = 0.0f; nz = 1.0f; }
	else { nx /= len; ny /= len; nz /= len; }
	P.ground_n[0] = nx; P.ground_n[1] = ny; P.ground_n[2] = nz;
	P.ground_on = enabled != 0;
	P.ground_h = isfinite(height) ? height : 0.0f;
	P.ground_fric = fmaxf(0.0f, friction);
	P.ground_rest = fminf(fmaxf(restitution, 0.0f), 1.0f);
	P.ground_radius = fmaxf(0.0f, contactRadius);
	P.ground_slop = fmaxf(0.0f, contactSlop);
	P.ground_gravity = fmaxf(0.0f, gravity);
}

/* setObjectModeParams(stiffness, no body contact, 50) (xpbd_capi.cu:148, forward.cu:4464-4477) */
EXPORT void xpbd_set_object_shape(float stiffness)
{
	float s = fminf(fmaxf(stiffness, 0.0f), 1.0f);
	if (!isfinite(s)) s = 0.0f;
	P.obj_shape = s;
}

/* setObjectShapeGPU (forward.cu:4521): the weighted fit while pinned (1) or the plain fit */
EXPORT void xpbd_set_object_shape_gpu(int enabled) { g_obj_gpu = enabled != 0; }

/* setKinematicColliders (forward.cu:4478-4500) */
EXPORT void xpbd_set_colliders(int count, const int* types, const float* poses, const float* dims, float margin,
	float friction)
{
	if (count < 0) count = 0;
	if (count > MAX_KIN) count = MAX_KIN;
	const int samePrev = (count == P.kin_count);
	for (int c = 0; c < count; ++c) {
		kin_t* K = &P.kin[c];
		const int keep = samePrev && K->type == types[c];
		for (int a = 0; a < 9; ++a) K->Rp[a] = keep ? K->R[a] : poses[12 * c + a];
		for (int a = 0; a < 3; ++a) K->tp[a] = keep ? K->t[a] : poses[12 * c + 9 + a];
		K->type = types[c];
		for (int a = 0; a < 9; ++a) K->R[a] = poses[12 * c + a];
		for (int a = 0; a < 3; ++a) { K->t[a] = poses[12 * c + 9 + a]; K->h[a] = fmaxf(dims[3 * c + a], 0.0f); }
	}
	P.kin_count = count;
	P.kin_margin = (isfinite(margin) && margin > 0.0f) ? margin : 0.0f;
	P.kin_friction = (isfinite(friction) && friction > 0.0f) ? friction : 0.0f;
}

/* getKinematicColliderStats (forward.cu:4502-4519) */
EXPORT int xpbd_collider_stats(int* hits, float* push, float* centroid, int maxCount)
{
	const int n = maxCount < P.kin_count ? maxCount : P.kin_count;
	if (n <= 0 || !S.stepped) return 0;
	for (int c = 0; c < n; ++c) {
		if (hits) hits[c] = P.kin_hits[c];
		const float* a = &P.kin_push[KIN_ACC * c];
		for (int k = 0; k < 3; ++k) {
			if (push) push[3 * c + k] = a[k];
			if (centroid) centroid[3 * c + k] = (a[6] > 0.0f) ? a[3 + k] / a[6] : P.kin[c].t[k];
		}
	}
	return n;
}

/* addRigidVelocityAllKernel (forward.cu:6701-6712) */
EXPORT int xpbd_add_rigid_velocity(const float* dv, const float* dw, const float* center)
{
	if (!S.stepped) return fail("xpbd_add_rigid_velocity: no step yet");
	for (int idx = 0; idx < S.n; ++idx) {
		if (S.inv_mass[idx] <= 0.0f) continue;
		const f3 p = S.pos_curr[idx];
		const float rx = p.x - center[0], ry = p.y - center[1], rz = p.z - center[2];
		const f3 v = S.vel[idx];
		S.vel[idx] = mk3(v.x + dv[0] + (dw[1] * rz - dw[2] * ry), v.y + dv[1] + (dw[2] * rx - dw[0] * rz),
			v.z + dv[2] + (dw[0] * ry - dw[1] * rx));
	}
	return 0;
}

/* xpbd_set_contact_shape (xpbd_capi.cu:181-191): pack from the created shapes */
EXPORT int xpbd_set_contact_shape(int enabled, float tau, float radiusCap)
{
	if (!S.created) return fail("xpbd_set_contact_shape: call xpbd_create first");
	S.contact_on = enabled != 0;
	S.contact_tau = tau;
	S.contact_cap = radiusCap;
	if (S.contact_on)
		contact_pack(S.scales, S.rots, S.opacity, S.n, tau, (isfinite(radiusCap) && radiusCap > 0.0f) ? radiusCap : 0.0f);
	S.contact_col = (enabled & 1) != 0;
	S.contact_ground = (enabled & 2) != 0;
	return 0;
}

/* setAttachedParticles + attachApplyKernel (forward.cu:6714-6725, 6759-6788) */
EXPORT int xpbd_set_attached(int count, const int* idx, const float* pos, float weight)
{
	if (!S.stepped) return fail("xpbd_set_attached: no step yet");
	const int N = S.n;
	if (S.att_active) memcpy(S.inv_mass, S.inv_mass_saved, sizeof(float) * N);
	if (count <= 0 || !idx || !pos) { S.att_active = 0; return 0; }
	if (!S.att_active) {
		if (!S.inv_mass_saved) S.inv_mass_saved = malloc(sizeof(float) * N);
		memcpy(S.inv_mass_saved, S.inv_mass, sizeof(float) * N);
	}
	/* rigid-fit weights of object mode: 1, pinned max(weight, 1) (forward.cu:6774, 6724) */
	if (!S.obj_w) S.obj_w = malloc(sizeof(float) * N);
	for (int i = 0; i < N; ++i) S.obj_w[i] = 1.0f;
	for (int k = 0; k < count; ++k) {
		const int i = idx[k];
		if (i < 0 || i >= N) continue;
		S.inv_mass[i] = 0.0f;
		S.pos_curr[i] = mk3(pos[3 * k], pos[3 * k + 1], pos[3 * k + 2]);
		S.vel[i] = mk3(0, 0, 0);
		S.obj_w[i] = fmaxf(weight, 1.0f);
	}
	S.att_active = 1;
	return 0;
}

/* setSelfCollisionParams (forward.cu:4532-4540) */
EXPORT void xpbd_set_self_collision(int enabled, float radiusScale, float excludeScale, int withinBody)
{
	P.sc_enabled = enabled != 0;
	P.sc_within = withinBody != 0;
	P.sc_radius_scale = fminf(fmaxf(isfinite(radiusScale) ? radiusScale : 1.5f, 0.1f), 10.0f);
	P.sc_exclude_scale = fminf(fmaxf(isfinite(excludeScale) ? excludeScale : 2.0f, 1.05f), 20.0f);
	if (!enabled) { S.sc_contacts = 0; S.sc_overflow = 0; }
}

EXPORT void xpbd_self_collision_stats(int* out)
{
	out[0] = S.sc_contacts;
	out[1] = S.sc_active;
	out[2] = S.sc_overflow;
}

EXPORT void xpbd_set_shape_robust(int enabled) { P.shape_robust = enabled != 0; }

EXPORT int xpbd_step(void)
{
	if (!S.created) return fail("xpbd_step: call xpbd_create first");
	ensure_built();
	run_step();
	S.stepped = 1;
	return 0;
}

EXPORT unsigned long long xpbd_positions_device(void) { return 0ull; }

EXPORT int xpbd_positions_host(float* out, int n)
{
	if (!S.stepped) return fail("xpbd_positions_host: no step yet");
	if (!out || n != S.n) return fail("xpbd_positions_host: size mismatch");
	memcpy(out, S.pos_curr, sizeof(float) * 3 * n);
	return 0;
}

/* symEig3Double (forward.cu:13022-13060) */
static void sym_eig3_double(double a[3][3], double ev[3], double V[3][3])
{
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c) V[r][c] = (r == c) ? 1.0 : 0.0;
	const int Pp[3] = { 0, 0, 1 }, Qq[3] = { 1, 2, 2 };
	for (int sweep = 0; sweep < 32; ++sweep) {
		const double off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
		const double diag = fabs(a[0][0]) + fabs(a[1][1]) + fabs(a[2][2]);
		if (off <= 1e-15 * diag + 1e-300) break;
		for (int k = 0; k < 3; ++k) {
			const int p = Pp[k], q = Qq[k];
			const double apq = a[p][q];
			if (fabs(apq) <= 1e-300) continue;
			const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
			const double t = ((theta >= 0.0) ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
			const double c = 1.0 / sqrt(t * t + 1.0);
			const double s = t * c;
			for (int m = 0; m < 3; ++m) {
				const double amp = a[m][p], amq = a[m][q];
				a[m][p] = c * amp - s * amq;
				a[m][q] = s * amp + c * amq;
			}
			for (int m = 0; m < 3; ++m) {
				const double apm = a[p][m], aqm = a[q][m];
				a[p][m] = c * apm - s * aqm;
				a[q][m] = s * apm + c * aqm;
			}
			for (int m = 0; m < 3; ++m) {
				const double vmp = V[m][p], vmq = V[m][q];
				V[m][p] = c * vmp - s * vmq;
				V[m][q] = s * vmp + c * vmq;
			}
		}
	}
	ev[0] = a[0][0]; ev[1] = a[1][1]; ev[2] = a[2][2];
}

/* deformedShapeKernel (forward.cu:13063-13225), robust path (forward.cu:4226) */
static int deformed_shape_node(int i, float deformEps, float* outScale, float* outQuat)
{
	const int N = S.n;
	const f3 s0 = mk3(S.scales[3 * i], S.scales[3 * i + 1], S.scales[3 * i + 2]);
	const float q0x = S.rots[4 * i], q0y = S.rots[4 * i + 1], q0z = S.rots[4 * i + 2], q0w = S.rots[4 * i + 3];
	const f3 x = S.pos_curr[i], x0 = S.pos_rest[i];
	const float dxv = x.x - x0.x, dyv = x.y - x0.y, dzv = x.z - x0.z;
	const float diff = sqrtf(dxv * dxv + dyv * dyv + dzv * dzv);
	const int kn = S.cnt[i];
	int deformed = 0;
	m3 Sigma = m3_zero();
	if (diff > deformEps && kn >= 3) {
		const int off = S.off[i];
		m3 PPt = m3_zero(), QPt = m3_zero();
		for (int k = 0; k < kn; ++k) {
			const int j = S.nbr[off + k];
			if (j < 0 || j >= N) continue;
			const f3 p = mk3(S.pos_rest[j].x - x0.x, S.pos_rest[j].y - x0.y, S.pos_rest[j].z - x0.z);
			const f3 q = mk3(S.pos_curr[j].x - x.x, S.pos_curr[j].y - x.y, S.pos_curr[j].z - x.z);
			m3_add_outer(&PPt, p, p);
			m3_add_outer(&QPt, q, p);
		}
		const float tracePPt = PPt.m[0][0] + PPt.m[1][1] + PPt.m[2][2];
		const float alpha = (tracePPt > 0.0f) ? (tracePPt * 1e-4f) : 1e-6f;
		m3 Dg = m3_diag(alpha);
		PPt = m3_addm(&PPt, &Dg);
		QPt = m3_addm(&QPt, &Dg);
		const float sP = fmaxf((PPt.m[0][0] + PPt.m[1][1] + PPt.m[2][2]) * (1.0f / 3.0f), 1e-30f);
		const float invSP = 1.0f / sP;
		m3 invHat, invPPt;
		m3 Ph = m3_scale(&PPt, invSP);
		const int ok = inverse3x3_safe(&Ph, &invHat, 1e-9f);
		if (ok) {
			invPPt = m3_scale(&invHat, invSP);
			const m3 A = m3_mul(&QPt, &invPPt);
			const m3 At = m3_transpose(&A);
			const m3 AtA = m3_mul(&At, &A);
			m3 V;
			f3 S2;
			eig_glm(&AtA, &S2, &V);
			f3 Sv = mk3(sqrtf(fmaxf(0.0f, S2.x)), sqrtf(fmaxf(0.0f, S2.y)), sqrtf(fmaxf(0.0f, S2.z)));
			Sv = mk3(fminf(fmaxf(Sv.x, 1e-3f), 1.5f), fminf(fmaxf(Sv.y, 1e-3f), 1.5f), fminf(fmaxf(Sv.z, 1e-3f), 1.5f));
			const float eps = 1.0e-7f;
			m3 Si = m3_zero();
			Si.m[0][0] = (Sv.x > eps) ? 1.0f / Sv.x : 0.0f;
			Si.m[1][1] = (Sv.y > eps) ? 1.0f / Sv.y : 0.0f;
			Si.m[2][2] = (Sv.z > eps) ? 1.0f / Sv.z : 0.0f;
			const m3 AV = m3_mul(&A, &V);
			m3 U = m3_mul(&AV, &Si);
			const m3 Vt = m3_transpose(&V);
			m3 R = m3_mul(&U, &Vt);
			if (m3_det(&R) < 0.0f) {
				U.m[0][0] *= -1.0f; U.m[0][1] *= -1.0f; U.m[0][2] *= -1.0f;
				R = m3_mul(&U, &Vt);
			}
			m3 Sd = m3_zero();
			Sd.m[0][0] = Sv.x; Sd.m[1][1] = Sv.y; Sd.m[2][2] = Sv.z;
			const m3 VS = m3_mul(&V, &Sd);
			const m3 S_final = m3_mul(&VS, &Vt);
			m3 Sm = m3_diag(1.0f);
			Sm.m[0][0] = s0.x; Sm.m[1][1] = s0.y; Sm.m[2][2] = s0.z;
			const float r = q0x, qx = q0y, qy = q0z, qz = q0w;
			m3 R0;
			R0.m[0][0] = 1.f - 2.f * (qy * qy + qz * qz); R0.m[0][1] = 2.f * (qx * qy - r * qz);
			R0.m[0][2] = 2.f * (qx * qz + r * qy);
			R0.m[1][0] = 2.f * (qx * qy + r * qz); R0.m[1][1] = 1.f - 2.f * (qx * qx + qz * qz);
			R0.m[1][2] = 2.f * (qy * qz - r * qx);
			R0.m[2][0] = 2.f * (qx * qz - r * qy); R0.m[2][1] = 2.f * (qy * qz + r * qx);
			R0.m[2][2] = 1.f - 2.f * (qx * qx + qy * qy);
			const m3 SR0 = m3_mul(&Sm, &R0);
			const m3 SR0S = m3_mul(&SR0, &S_final);
			const m3 Rt = m3_transpose(&R);
			const m3 M = m3_mul(&SR0S, &Rt);
			const m3 Mt = m3_transpose(&M);
			Sigma = m3_mul(&Mt, &M);
			deformed = m3_finite(&Sigma);
		}
	}
	const double tr = deformed ? ((double)Sigma.m[0][0] + Sigma.m[1][1] + Sigma.m[2][2]) : 0.0;
	if (!deformed || !(tr > 0.0)) {
		outScale[0] = s0.x; outScale[1] = s0.y; outScale[2] = s0.z;
		outQuat[0] = q0x; outQuat[1] = q0y; outQuat[2] = q0z; outQuat[3] = q0w;
		return 0;
	}
	const double inv = 3.0 / tr;
	double a[3][3];
	for (int rr = 0; rr < 3; ++rr)
		for (int c = 0; c < 3; ++c) a[rr][c] = 0.5 * ((double)Sigma.m[c][rr] + (double)Sigma.m[rr][c]) * inv;
	double ev[3], E[3][3];
	sym_eig3_double(a, ev, E);
	const double det = E[0][0] * (E[1][1] * E[2][2] - E[1][2] * E[2][1])
		- E[0][1] * (E[1][0] * E[2][2] - E[1][2] * E[2][0])
		+ E[0][2] * (E[1][0] * E[2][1] - E[1][1] * E[2][0]);
	if (det < 0.0)
		for (int rr = 0; rr < 3; ++rr) E[rr][2] = -E[rr][2];
	const double sFloor = 1e-3 * (double)fmaxf(s0.x, fmaxf(s0.y, s0.z));
	for (int k = 0; k < 3; ++k) outScale[k] = (float)fmax(sqrt(fmax(ev[k], 0.0) / inv), sFloor);
	double w, qxv, qyv, qzv;
	const double t = E[0][0] + E[1][1] + E[2][2];
	if (t > 0.0) {
		const double s = 2.0 * sqrt(t + 1.0);
		w = 0.25 * s; qxv = (E[2][1] - E[1][2]) / s; qyv = (E[0][2] - E[2][0]) / s; qzv = (E[1][0] - E[0][1]) / s;
	}
	else if (E[0][0] > E[1][1] && E[0][0] > E[2][2]) {
		const double s = 2.0 * sqrt(1.0 + E[0][0] - E[1][1] - E[2][2]);
		w = (E[2][1] - E[1][2]) / s; qxv = 0.25 * s; qyv = (E[0][1] + E[1][0]) / s; qzv = (E[0][2] + E[2][0]) / s;
	}
	else if (E[1][1] > E[2][2]) {
		const double s = 2.0 * sqrt(1.0 + E[1][1] - E[0][0] - E[2][2]);
		w = (E[0][2] - E[2][0]) / s; qxv = (E[0][1] + E[1][0]) / s; qyv = 0.25 * s; qzv = (E[1][2] + E[2][1]) / s;
	}
	else {
		const double s = 2.0 * sqrt(1.0 + E[2][2] - E[0][0] - E[1][1]);
		w = (E[1][0] - E[0][1]) / s; qxv = (E[0][2] + E[2][0]) / s; qyv = (E[1][2] + E[2][1]) / s; qzv = 0.25 * s;
	}
	const double qn = sqrt(w * w + qxv * qxv + qyv * qyv + qzv * qzv);
	outQuat[0] = (float)(w / qn);
	outQuat[1] = (float)(qxv / qn);
	outQuat[2] = (float)(qyv / qn);
	outQuat[3] = (float)(qzv / qn);
	return 1;
}

EXPORT int xpbd_compute_shapes(float deformEps, float* hostScales, float* hostQuats, int n)
{
	if (!S.stepped) return fail("xpbd_compute_shapes: no step yet");
	if (n != S.n) return fail("xpbd_compute_shapes: size mismatch");
	float* sc = malloc(sizeof(float) * 3 * n);
	float* qt = malloc(sizeof(float) * 4 * n);
	int deformed = 0;
#pragma omp parallel for schedule(static) reduction(+ : deformed) num_threads(nthreads())
	for (int i = 0; i < n; ++i) deformed += deformed_shape_node(i, deformEps, sc + 3 * i, qt + 4 * i);
	/* contact ellipsoids follow the deformed shapes from the next step (xpbd_capi.cu:255-256) */
	if (S.contact_on)
		contact_pack(sc, qt, S.opacity, n, S.contact_tau,
			(isfinite(S.contact_cap) && S.contact_cap > 0.0f) ? S.contact_cap : 0.0f);
	if (hostScales) memcpy(hostScales, sc, sizeof(float) * 3 * n);
	if (hostQuats) memcpy(hostQuats, qt, sizeof(float) * 4 * n);
	free(sc);
	free(qt);
	return deformed;
}

/* xpbd_reset (capi:263-269) -> setAttachedParticles(0) + squashReset (forward.cu:4411-4427) */
EXPORT int xpbd_reset(void)
{
	if (!S.stepped) return fail("xpbd_reset: no step yet");
	Q.active = 0; Q.cur = 0.0f; Q.ckpt = 0; Q.dwell = 0;   /* squashReset (forward.cu:4411-4427) */
	if (S.att_active) memcpy(S.inv_mass, S.inv_mass_saved, sizeof(float) * S.n);
	S.att_active = 0;
	memcpy(S.pos_curr, S.pos_rest, sizeof(f3) * S.n);
	memset(S.vel, 0, sizeof(f3) * S.n);
	for (int i = 0; i < S.n; ++i) S.inv_mass[i] = 1.0f;
	memset(S.lam_vol, 0, sizeof(float) * S.n);
	return 0;
}

/* groundLaunch (forward.cu:4551-4610) */
EXPORT int xpbd_launch(const float* lin, const float* ang, const float* tilt)
{
	if (!S.stepped) return fail("xpbd_launch: no step yet");
	Q.active = 0; Q.cur = 0.0f; Q.ckpt = 0; Q.dwell = 0;   /* groundLaunch ends a press (forward.cu:4599-4602) */
	const int N = S.n;
	double cx = 0.0, cy = 0.0, cz = 0.0;
	for (int i = 0; i < N; ++i) { cx += S.pos_rest[i].x; cy += S.pos_rest[i].y; cz += S.pos_rest[i].z; }
	const float comX = (float)(cx / N), comY = (float)(cy / N), comZ = (float)(cz / N);
	const float ax = tilt ? tilt[0] : 0.0f, ay = tilt ? tilt[1] : 0.0f, az = tilt ? tilt[2] : 0.0f;
	const float th = sqrtf(ax * ax + ay * ay + az * az);
	float R[9] = { 1, 0, 0, 0, 1, 0, 0, 0, 1 };
	if (th > 1e-8f) {
		const float kx = ax / th, ky = ay / th, kz = az / th;
		const float s = sinf(th), c = cosf(th), t = 1.0f - c;
		R[0] = c + t * kx * kx; R[1] = t * kx * ky - s * kz; R[2] = t * kx * kz + s * ky;
		R[3] = t * ky * kx + s * kz; R[4] = c + t * ky * ky; R[5] = t * ky * kz - s * kx;
		R[6] = t * kz * kx - s * ky; R[7] = t * kz * ky + s * kx; R[8] = c + t * kz * kz;
	}
	const float vx = lin ? lin[0] : 0.0f, vy = lin ? lin[1] : 0.0f, vz = lin ? lin[2] : 0.0f;
	const float wx = ang ? ang[0] : 0.0f, wy = ang ? ang[1] : 0.0f, wz = ang ? ang[2] : 0.0f;
	for (int i = 0; i < N; ++i) {
		const float px = S.pos_rest[i].x - comX, py = S.pos_rest[i].y - comY, pz = S.pos_rest[i].z - comZ;
		const float rx = R[0] * px + R[1] * py + R[2] * pz;
		const float ry = R[3] * px + R[4] * py + R[5] * pz;
		const float rz = R[6] * px + R[7] * py + R[8] * pz;
		S.pos_curr[i] = mk3(comX + rx, comY + ry, comZ + rz);
		S.vel[i] = mk3(vx + (wy * rz - wz * ry), vy + (wz * rx - wx * rz), vz + (wx * ry - wy * rx));
		S.inv_mass[i] = 1.0f;
	}
	memset(S.lam_vol, 0, sizeof(float) * N);
	return 0;
}

/* xpbd_press_start (capi:281-288) -> squashStart in press mode (forward.cu:4311-4396) */
EXPORT int xpbd_press_start(int axis, float rampPerSec, float maxDispPct, int fromLo)
{
	if (!S.stepped) return fail("xpbd_press_start: step once first");
	if (axis < 0 || axis > 2) axis = 1;
	const float slab = 0.08f;
	maxDispPct = fmaxf(0.01f, fminf(1.0f, maxDispPct));
	float lo = FLT_MAX, hi = -FLT_MAX;
	for (int i = 0; i < S.n; ++i) {
		const float v = S.pos_in[3 * i + axis];
		lo = fminf(lo, v);
		hi = fmaxf(hi, v);
	}
	const float extent = hi - lo;
	const float top = hi - slab * extent, bot = lo + slab * extent;
	int ntop = 0, nbot = 0;
	for (int i = 0; i < S.n; ++i) {
		const float v = S.pos_in[3 * i + axis];
		if (v >= top) ++ntop; else if (v <= bot) ++nbot;
	}
	if (ntop == 0 || nbot == 0) return fail("xpbd_press_start: squashStart failed");
	Q.axis = axis; Q.ramp = rampPerSec; Q.lo = lo; Q.hi = hi; Q.max = maxDispPct * extent;
	Q.from_lo = fromLo != 0; Q.cur = 0.0f; Q.ckpt = 0; Q.dwell = 0; Q.active = 1;
	return 0;
}
EXPORT void xpbd_press_autolog(int enabled) { Q.autolog = enabled != 0; }
/* squashStop (forward.cu:4398-4409) */
EXPORT void xpbd_press_stop(void)
{
	if (!Q.active) return;
	Q.active = 0;
	for (int i = 0; i < S.n && S.inv_mass; ++i) S.inv_mass[i] = 1.0f;
}
/* squashGetProgress + squashGetPlates (forward.cu:4675-4689) */
EXPORT int xpbd_press_state(float* lo, float* hi, float* cur, float* mx)
{
	if (cur) *cur = Q.cur;
	if (mx) *mx = Q.max;
	if (lo) *lo = Q.lo + ((Q.active && Q.from_lo) ? Q.cur : 0.0f);
	if (hi) *hi = Q.hi - ((Q.active && !Q.from_lo) ? Q.cur : 0.0f);
	return Q.active ? 1 : 0;
}

/* setVolumeJStatsEnabled + getVolumeJVolumeWeighted (forward.cu:4081-4099) */
EXPORT void xpbd_volume_stats(int enable, float* jvw, float* jvwStd)
{
	P.jstats = enable != 0;
	if (jvw) *jvw = S.jvw_mean;
	if (jvwStd) *jvwStd = S.jvw_std;
}

/* ------------------------------------------------------------------------- */
/* oracle-only accessors                                                      */
/* ------------------------------------------------------------------------- */
EXPORT void oracle_set_gs(int distance, int volume) { P.dist_gs = distance != 0; P.vol_gs = volume != 0; }
/* current positions from the caller (float3[n]), velocities kept: lets a test run the
 * deformed-shape writeback on positions another solver produced */
EXPORT int oracle_set_positions(const float* pos, int n)
{
	if (!S.stepped || !pos || n != S.n) return fail("oracle_set_positions: no step yet or size mismatch");
	for (int i = 0; i < n; ++i) S.pos_curr[i] = mk3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
	return 0;
}
EXPORT void oracle_set_volume_warp_mode(int mode) { P.warp_mode = mode; }
EXPORT void oracle_set_threads(int n) { P.threads = n > 0 ? n : 0; }
EXPORT int oracle_get_threads(void) { return nthreads(); }

EXPORT void oracle_sizes(long long* out)
{
	out[0] = S.n;
	out[1] = S.m;
	out[2] = S.vol_total;
	out[3] = S.rev_total;
	out[4] = S.gs_nedges;
	out[5] = S.gs_ncolors;
	out[6] = S.vol_gs_clusters;
	out[7] = S.vol_gs_ncolors;
	out[8] = S.sc_table;
	out[9] = S.sc_contacts;
}

static int copy_i(const int* src, long long n, int* out, long long cap)
{
	if (!src || n < 0) return -1;
	if (!out) return (int)n;
	if (cap < n) return -1;
	memcpy(out, src, sizeof(int) * (size_t)n);
	return (int)n;
}
static int copy_f(const float* src, long long n, float* out, long long cap)
{
	if (!src || n < 0) return -1;
	if (!out) return (int)n;
	if (cap < n) return -1;
	memcpy(out, src, sizeof(float) * (size_t)n);
	return (int)n;
}

EXPORT int oracle_int(const char* name, int* out, long long cap)
{
	const int N = S.n;
	if (!strcmp(name, "vol_offset")) return copy_i(S.vol_off, N, out, cap);
	if (!strcmp(name, "vol_count")) return copy_i(S.vol_cnt, N, out, cap);
	if (!strcmp(name, "vol_idx")) return copy_i(S.vol_idx, S.vol_total, out, cap);
	if (!strcmp(name, "rev_offset")) return copy_i(S.rev_off, N, out, cap);
	if (!strcmp(name, "rev_count")) return copy_i(S.rev_cnt, N, out, cap);
	if (!strcmp(name, "rev_idx")) return copy_i(S.rev_idx, S.rev_total, out, cap);
	if (!strcmp(name, "mat_type")) return copy_i(S.mat_type, N, out, cap);
	if (!strcmp(name, "nbr_offset")) return copy_i(S.off, N, out, cap);
	if (!strcmp(name, "nbr_count")) return copy_i(S.cnt, N, out, cap);
	if (!strcmp(name, "nbr_idx")) return copy_i(S.nbr, S.m, out, cap);
	if (!strcmp(name, "gs_edge")) return copy_i(S.gs_edge, 2LL * S.gs_nedges, out, cap);
	if (!strcmp(name, "gs_color_offset")) return copy_i(S.gs_color_off, S.gs_color_off ? S.gs_ncolors + 1 : -1, out, cap);
	if (!strcmp(name, "vol_gs_order")) return copy_i(S.vol_gs_order, S.vol_gs_clusters, out, cap);
	if (!strcmp(name, "vol_gs_color_offset"))
		return copy_i(S.vol_gs_color_off, S.vol_gs_color_off ? S.vol_gs_ncolors + 1 : -1, out, cap);
	if (!strcmp(name, "sc_keys")) return copy_i((const int*)S.sc_keys, N, out, cap);
	if (!strcmp(name, "sc_keys_sorted")) return copy_i((const int*)S.sc_keys_sorted, N, out, cap);
	if (!strcmp(name, "sc_idx_sorted")) return copy_i(S.sc_idx_sorted, N, out, cap);
	if (!strcmp(name, "sc_cell_start")) return copy_i(S.sc_cell_start, S.sc_table, out, cap);
	if (!strcmp(name, "sc_cell_end")) return copy_i(S.sc_cell_end, S.sc_table, out, cap);
	if (!strcmp(name, "sc_contact")) return copy_i(S.sc_contact, (long long)N * SC_MAX, out, cap);
	if (!strcmp(name, "sc_count")) return copy_i(S.sc_count, N, out, cap);
	if (!strcmp(name, "obj_id")) return copy_i(S.obj_id, N, out, cap);
	return -1;
}

EXPORT int oracle_float(const char* name, float* out, long long cap)
{
	const int N = S.n;
	if (!strcmp(name, "det_rest")) return copy_f(S.det_rest, N, out, cap);
	if (!strcmp(name, "sigma_rest")) return copy_f(S.sigma_rest, 6LL * N, out, cap);
	if (!strcmp(name, "v_rest")) return copy_f(S.v_rest, N, out, cap);
	if (!strcmp(name, "rest_len")) return copy_f(S.rest_len, N, out, cap);
	if (!strcmp(name, "gs_rest")) return copy_f(S.gs_rest, S.gs_nedges, out, cap);
	if (!strcmp(name, "gs_stiff")) return copy_f(S.gs_stiff, S.gs_nedges, out, cap);
	if (!strcmp(name, "vel")) return copy_f((const float*)S.vel, 3LL * N, out, cap);
	if (!strcmp(name, "pos_rest")) return copy_f((const float*)S.pos_rest, 3LL * N, out, cap);
	if (!strcmp(name, "pos_next")) return copy_f((const float*)S.pos_next, 3LL * N, out, cap);
	if (!strcmp(name, "inv_mass")) return copy_f(S.inv_mass, N, out, cap);
	if (!strcmp(name, "cluster_coef")) return copy_f(S.cl_coef, N, out, cap);
	if (!strcmp(name, "self_col")) {
		if (!out) return 3;
		if (cap < 3) return -1;
		out[0] = S.sc_spacing;
		out[1] = P.sc_radius_scale * S.sc_spacing;
		out[2] = S.sc_reach;
		return 3;
	}
	return -1;
}

/* ------------------------------------------------------------------------- */
/* ChainMail displacement propagation (runChainmailGPU, forward.cu:12808-13006, */
/* the dense path: no active map, no inertia)                                 */
/* ------------------------------------------------------------------------- */
/* material controls (forward.cu:66-71 defaults, setChainmailMaterialParams 4844-4858) */
static struct {
	float global, air, skin, bone, influence;
	int use_edge;
} CM = { 1.0f, 0.1f, 0.1f, 0.1f, 1.0f, 1 };

#define CM_AIR 0.13f   /* forward.h:63-65 */
#define CM_SKIN 0.45f
#define CM_BONE 0.75f

/* cm_getConstraint (forward.cu:5221-5264): the axis tolerance of a density class */
static float cm_axis_tol(float density)
{
	float c;
	if (density < CM_AIR) c = CM.air;
	else if (density < CM_SKIN) c = CM.skin;
	else c = CM.bone;
	const float scale = fmaxf(1e-4f, CM.global);
	return c * scale;
}

/* cm_edgeScaleFromStiff (forward.cu:5266-5278) */
static float cm_edge_scale(float stiff)
{
	if (!CM.use_edge || CM.influence <= 0.0f) return 1.0f;
	const float s = fminf(fmaxf(stiff, 0.05f), 1.0f);
	const float t = (s - 0.05f) / 0.95f;
	const float scale = 1.0f + CM.influence * (t * 2.0f - 1.0f);
	return fminf(fmaxf(scale, 0.1f), 4.0f);
}

/* cm_propagationTime (forward.cu:5280-5293) */
static float cm_link_time(float d0, float d1)
{
	float et, nt;
	if (d0 < CM_AIR) et = 1.0f;
	else if (d0 < CM_SKIN) et = 0.3f;
	else if (d0 < CM_BONE) et = 0.05f;
	else et = 0.005f;
	if (d1 < CM_AIR) nt = 1.0f;
	else if (d1 < CM_SKIN) nt = 0.3f;
	else if (d1 < CM_BONE) nt = 0.05f;
	else nt = 0.005f;
	return (et + nt) * 0.5f;
}

/* cm_correctionFromNeighbor (forward.cu:5295-5330) */
static f3 cm_correction(f3 epos, f3 npos, float targ, float ndens, float stiff)
{
	const float dx = cm_axis_tol(ndens);
	const float edge_scale = cm_edge_scale(stiff);
	const f3 dir = f3_sub(epos, npos);
	const float len = f3_len(dir);
	if (len < 1e-6f) return mk3(0.0f, 0.0f, 0.0f);
	const float inv_len = 1.0f / len;
	const f3 nd = f3_mul(dir, inv_len);
	if (len < targ - dx) {
		const float delta = (targ - dx) - len;
		return f3_mul(nd, delta * edge_scale);
	}
	if (len > targ + dx) {
		const float delta = len - (targ + dx);
		return f3_mul(nd, -(delta * edge_scale));
	}
	return mk3(0.0f, 0.0f, 0.0f);
}

/* chainmailPropagateKernelBest (forward.cu:5396-5464): the fastest neighbour only */
static void cm_propagate(const f3* pin, f3* pout, const float* tin, float* tout, float strength)
{
#pragma omp parallel for schedule(static) num_threads(nthreads())
	for (int i = 0; i < S.n; ++i) {
		const f3 epos = pin[i];
		const float edens = S.density[i];
		const float tcur = tin[i];
		float best_time = tcur, best_dist = 0.0f, best_dens = 0.0f;
		int best = -1;
		const int off = S.off[i], cnt = S.cnt[i];
		for (int k = 0; k < cnt; ++k) {
			const int j = S.nbr[off + k];
			const float nd = S.density[j];
			const float cand = tin[j] + cm_link_time(edens, nd);
			if (cand < best_time) { best_time = cand; best = j; best_dist = S.ndist[off + k]; best_dens = nd; }
		}
		f3 out = epos;
		if (best >= 0 && best_time < tcur) {
			float stiff = 1.0f;
			for (int k = 0; k < cnt; ++k)
				if (S.nbr[off + k] == best) { stiff = S.nstiff[off + k]; break; }
			const f3 corr = cm_correction(epos, pin[best], best_dist, best_dens, stiff);
			if (f3_len(corr) > 0.0f) out = f3_add(epos, f3_mul(corr, strength));
		}
		pout[i] = out;
		tout[i] = best_time;
	}
}

/* chainmailRelaxKernel (forward.cu:5466-5559) */
static void cm_relax(const f3* pin, f3* pout, float stiffness, float damping)
{
#pragma omp parallel for schedule(static) num_threads(nthreads())
	for (int i = 0; i < S.n; ++i) {
		const f3 epos = pin[i];
		const float etol = cm_axis_tol(S.density[i]);
		f3 acc = mk3(0.0f, 0.0f, 0.0f);
		int corr_count = 0, dist_count = 0;
		float sum_target = 0.0f;
		const int off = S.off[i], cnt = S.cnt[i];
		for (int k = 0; k < cnt; ++k) {
			const int j = S.nbr[off + k];
			const f3 npos = pin[j];
			const float ntol = cm_axis_tol(S.density[j]);
			const float edge_scale = cm_edge_scale(S.nstiff[off + k]);
			const float targ = S.ndist[off + k];
			const float tol = (0.0000001f * (etol + ntol)) / edge_scale;
			const f3 dir = f3_sub(npos, epos);
			const float len = f3_len(dir);
			if (len < 1e-6f) continue;
			const float inv_len = 1.0f / len;
			const f3 nd = f3_mul(dir, inv_len);
			if (len < targ - tol) {
				const float delta = (targ - tol) - len;
				acc = f3_sub(acc, f3_mul(nd, delta * edge_scale));
				corr_count++;
			}
			else if (len > targ + tol) {
				const float delta = len - (targ + tol);
				acc = f3_add(acc, f3_mul(nd, delta * edge_scale));
				corr_count++;
			}
			sum_target += targ;
			dist_count++;
		}
		if (corr_count > 0) {
			f3 avg = f3_mul(acc, 1.0f / (float)corr_count);
			float max_step = 0.6f;
			if (dist_count > 0) max_step = 1.5f * (sum_target / (float)dist_count);
			const float cl = f3_len(avg);
			if (cl > 1e-6f && cl > max_step) avg = f3_mul(avg, max_step / cl);
			const f3 corrected = f3_add(epos, f3_mul(avg, stiffness));
			pout[i] = f3_add(epos, f3_mul(f3_sub(corrected, epos), 1.0f - damping));
		}
		else {
			pout[i] = epos;
		}
	}
}

EXPORT void oracle_chainmail_set_material(float global_scale, float air, float skin, float bone, int use_edge_stiffness,
	float edge_influence)
{
	CM.global = fmaxf(1e-4f, global_scale);
	CM.air = fmaxf(1e-4f, air);
	CM.skin = fmaxf(1e-4f, skin);
	CM.bone = fmaxf(1e-4f, bone);
	CM.use_edge = use_edge_stiffness != 0;
	CM.influence = fmaxf(0.0f, edge_influence);
}

/* applySeedCommandsKernel (forward.cu:5907-5924): seeds move by delta and start the wave
 * (arrival time 0); applied in order */
EXPORT int oracle_chainmail_seed(int count, const int* idx, const float* delta)
{
	if (!S.stepped) return fail("oracle_chainmail_seed: no step yet");
	if (count < 0 || (count > 0 && (!idx || !delta))) return fail("oracle_chainmail_seed: invalid arguments");
	for (int k = 0; k < count; ++k)
		if (idx[k] < 0 || idx[k] >= S.n) return fail("oracle_chainmail_seed: index out of range");
	for (int k = 0; k < count; ++k) {
		const int id = idx[k];
		S.pos_curr[id] = f3_add(S.pos_curr[id], mk3(delta[3 * k], delta[3 * k + 1], delta[3 * k + 2]));
		S.cm_time[id] = 0.0f;
	}
	return 0;
}

/* runChainmailGPU dense path (forward.cu:12901-12999): prop_iters propagation sweeps,
 * relax_iters relax sweeps, then one more relax sweep */
EXPORT int oracle_chainmail_run(int prop_iters, int relax_iters, float prop_strength, float relax_stiffness,
	float relax_damping)
{
	if (!S.stepped) return fail("oracle_chainmail_run: no step yet");
	if (prop_iters < 0 || relax_iters < 0) return fail("oracle_chainmail_run: negative iteration count");
	for (int it = 0; it < prop_iters; ++it) {
		cm_propagate(S.pos_curr, S.pos_next, S.cm_time, S.cm_time_next, prop_strength);
		f3* t = S.pos_curr; S.pos_curr = S.pos_next; S.pos_next = t;
		float* u = S.cm_time; S.cm_time = S.cm_time_next; S.cm_time_next = u;
	}
	for (int it = 0; it <= relax_iters; ++it) {
		cm_relax(S.pos_curr, S.pos_next, relax_stiffness, relax_damping);
		f3* t = S.pos_curr; S.pos_curr = S.pos_next; S.pos_next = t;
	}
	return 0;
}

EXPORT int oracle_chainmail_times(float* out, int n)
{
	if (!S.built || !out || n < S.n) return fail("oracle_chainmail_times: invalid arguments");
	memcpy(out, S.cm_time, sizeof(float) * S.n);
	return S.n;
}

EXPORT int oracle_selfcol_build(const float* x, const float* p)
{
	if (!S.built || !x || !p) return -1;
	memcpy(S.pos_curr, x, sizeof(f3) * S.n);
	memcpy(S.pos_next, p, sizeof(f3) * S.n);
	sc_build(S.pos_curr, S.pos_next);
	return S.sc_contacts;
}
