// sm_100a kernels of the XPBD Gaussian-graph step.
//
// Every kernel restates one stage of the reference step (runXPBDSimulation,
// forward.cu:12038-12751) with the same arithmetic order, so results stay within
// FP32 rounding of the reference; the data layout is this library's own (float4
// positions with the inverse mass in w, 36-byte blackboard records, CSR row starts with
// an N+1 sentinel, in-place distance multipliers).  None of these stages
// is a dense contraction, so none uses tensor cores; each is bounded by HBM or L2
// bandwidth (see the per-kernel notes).
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>

#include "xpbd_internal.h"

namespace xpbd {
namespace dev {

// ---------------------------------------------------------------------------
// small helpers (forward.cu:4949-4969; glm mat3 is column-major: m[col][row])
// ---------------------------------------------------------------------------
struct M3 { float m[3][3]; };

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 mul3(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float len3(float3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ bool fin3(float3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
__device__ __forceinline__ float comp(float3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
__device__ __forceinline__ float4 ld4(const float4* p, int i) { return __ldg(p + i); }
// Loads of data a kernel itself writes must not take the read-only (non-coherent) path:
// the fused substep kernel writes positions and cluster records in one phase and reads
// them in the next.  NC = true keeps __ldg where the data is constant for the launch.
// With NC = false the load is an explicit ld.global (coherent after a grid barrier), so
// that the compiler cannot turn a load through a const __restrict__ pointer into a
// read-only one.
template <bool NC> __device__ __forceinline__ float4 ldv(const float4* p, int i)
{
	if (NC) return __ldg(p + i);
	float4 v;
	asm volatile("ld.global.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p + i));
	return v;
}
template <bool NC> __device__ __forceinline__ float ldv(const float* p, int i)
{
	if (NC) return __ldg(p + i);
	float v;
	asm volatile("ld.global.f32 %0, [%1];" : "=f"(v) : "l"(p + i));
	return v;
}

__device__ __forceinline__ void m3_zero(M3& a)
{
#pragma unroll
	for (int c = 0; c < 3; ++c)
#pragma unroll
		for (int r = 0; r < 3; ++r) a.m[c][r] = 0.0f;
}
// A += outerProduct(p, q): O[c][r] = p[r] * q[c]
__device__ __forceinline__ void m3_add_outer(M3& A, float3 p, float3 q)
{
#pragma unroll
	for (int c = 0; c < 3; ++c)
#pragma unroll
		for (int r = 0; r < 3; ++r) A.m[c][r] += comp(p, r) * comp(q, c);
}
__device__ __forceinline__ float3 m3_mulv(const M3& M, float3 v)
{
	return make_float3(M.m[0][0] * v.x + M.m[1][0] * v.y + M.m[2][0] * v.z,
		M.m[0][1] * v.x + M.m[1][1] * v.y + M.m[2][1] * v.z,
		M.m[0][2] * v.x + M.m[1][2] * v.y + M.m[2][2] * v.z);
}
__device__ __forceinline__ M3 m3_mul(const M3& A, const M3& B)
{
	M3 R;
#pragma unroll
	for (int c = 0; c < 3; ++c)
#pragma unroll
		for (int r = 0; r < 3; ++r)
			R.m[c][r] = A.m[0][r] * B.m[c][0] + A.m[1][r] * B.m[c][1] + A.m[2][r] * B.m[c][2];
	return R;
}
__device__ __forceinline__ M3 m3_t(const M3& M)
{
	M3 T;
#pragma unroll
	for (int c = 0; c < 3; ++c)
#pragma unroll
		for (int r = 0; r < 3; ++r) T.m[c][r] = M.m[r][c];
	return T;
}
__device__ __forceinline__ float m3_det(const M3& M)
{
	const float(*m)[3] = M.m;
	return +m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2])
		- m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2])
		+ m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
}
__device__ __forceinline__ bool m3_finite(const M3& M)
{
	bool ok = true;
#pragma unroll
	for (int c = 0; c < 3; ++c)
#pragma unroll
		for (int r = 0; r < 3; ++r) ok = ok && isfinite(M.m[c][r]);
	return ok;
}

// adjugate inverse with an absolute determinant floor (forward.cu:1696-1719)
__device__ __forceinline__ bool inverse3x3_safe(const M3& M, M3& inv, float eps_det)
{
	const float(*m)[3] = M.m;
	const float a00 = m[0][0], a01 = m[0][1], a02 = m[0][2];
	const float a10 = m[1][0], a11 = m[1][1], a12 = m[1][2];
	const float a20 = m[2][0], a21 = m[2][1], a22 = m[2][2];
	const float det = a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) + a02 * (a10 * a21 - a11 * a20);
	if (fabsf(det) < eps_det) return false;
	const float invdet = 1.0f / det;
	inv.m[0][0] = (a11 * a22 - a12 * a21) * invdet;
	inv.m[0][1] = -(a01 * a22 - a02 * a21) * invdet;
	inv.m[0][2] = (a01 * a12 - a02 * a11) * invdet;
	inv.m[1][0] = -(a10 * a22 - a12 * a20) * invdet;
	inv.m[1][1] = (a00 * a22 - a02 * a20) * invdet;
	inv.m[1][2] = -(a00 * a12 - a02 * a10) * invdet;
	inv.m[2][0] = (a10 * a21 - a11 * a20) * invdet;
	inv.m[2][1] = -(a00 * a21 - a01 * a20) * invdet;
	inv.m[2][2] = (a00 * a11 - a01 * a10) * invdet;
	return true;
}

// cyclic-max float Jacobi, ascending eigenvalues, eigenvectors as glm columns
// (jacobiEigenDecomposition3x3 + eigenDecomposition_glm, forward.cu:782-901)
__device__ __noinline__ void eig_sym3f(const M3& Ag, float3& evals, M3& evecs)
{
	float A[3][3], V[3][3];
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) { A[r][c] = Ag.m[c][r]; V[r][c] = (r == c) ? 1.0f : 0.0f; }
	for (int iter = 0; iter < 50; ++iter) {
		int p = 0, q = 1;
		float maxOff = fabsf(A[0][1]);
		if (fabsf(A[0][2]) > maxOff) { p = 0; q = 2; maxOff = fabsf(A[0][2]); }
		if (fabsf(A[1][2]) > maxOff) { p = 1; q = 2; maxOff = fabsf(A[1][2]); }
		if (maxOff < 1e-6f) break;
		const float app = A[p][p], aqq = A[q][q], apq = A[p][q];
		const float phi = 0.5f * (aqq - app) / (apq + 1e-20f);
		const float t = (phi >= 0.0f) ? (1.0f / (phi + sqrtf(1.0f + phi * phi))) : (1.0f / (phi - sqrtf(1.0f + phi * phi)));
		const float c = 1.0f / sqrtf(1.0f + t * t);
		const float s = t * c;
		A[p][p] = app - t * apq;
		A[q][q] = aqq + t * apq;
		A[p][q] = A[q][p] = 0.0f;
		const int r = 3 - p - q;
		const float arp = A[r][p], arq = A[r][q];
		A[r][p] = A[p][r] = c * arp - s * arq;
		A[r][q] = A[q][r] = c * arq + s * arp;
#pragma unroll
		for (int rr = 0; rr < 3; ++rr) {
			const float vrp = V[rr][p], vrq = V[rr][q];
			V[rr][p] = c * vrp - s * vrq;
			V[rr][q] = s * vrp + c * vrq;
		}
	}
	float ev[3] = { A[0][0], A[1][1], A[2][2] };
#pragma unroll
	for (int i = 0; i < 2; ++i)
#pragma unroll
		for (int j = i + 1; j < 3; ++j)
			if (ev[i] > ev[j]) {
				const float te = ev[i]; ev[i] = ev[j]; ev[j] = te;
#pragma unroll
				for (int rr = 0; rr < 3; ++rr) { const float tv = V[rr][i]; V[rr][i] = V[rr][j]; V[rr][j] = tv; }
			}
	evals = make_float3(ev[0], ev[1], ev[2]);
#pragma unroll
	for (int c = 0; c < 3; ++c)
#pragma unroll
		for (int rr = 0; rr < 3; ++rr) evecs.m[c][rr] = V[rr][c];
}

// Sigma = s * SigmaHat, s = trace/3 (forward.cu:7666-7676)
__device__ __forceinline__ bool sigma_scale_det(const M3& S, float& scale, float& det_hat)
{
	const float s = (S.m[0][0] + S.m[1][1] + S.m[2][2]) * (1.0f / 3.0f);
	if (!isfinite(s) || s <= 1e-24f) return false;
	M3 H;
#pragma unroll
	for (int c = 0; c < 3; ++c)
#pragma unroll
		for (int r = 0; r < 3; ++r) H.m[c][r] = S.m[c][r] / s;
	const float d = m3_det(H);
	if (!isfinite(d) || d <= 1e-6f) return false;
	scale = s;
	det_hat = d;
	return true;
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

// ---------------------------------------------------------------------------
// ellipsoid contact shapes (forward.cu:7355-7399): each Gaussian meets colliders and
// the ground as its opacity-tau iso-ellipsoid, M = k^2 Sigma with k = sqrt(2 ln(a/tau)),
// instead of as its centre.  Stored per Gaussian in internal order as two float4,
// (xx, xy, xz, yy) and (yz, zz, -, -), beside the longest semi-axis rmax[i].
// ---------------------------------------------------------------------------
// support distance sqrt(n^T M n) along the unit normal n, summed as forward.cu:7387-7392
__device__ __forceinline__ float contact_support(float4 a, float4 b, float nx, float ny, float nz)
{
	const float q = a.x * nx * nx + a.w * ny * ny + b.y * nz * nz + 2.0f * (a.y * nx * ny + a.z * nx * nz + b.x * ny * nz);
	return sqrtf(fmaxf(q, 0.0f));
}

// contactShapePackKernel (forward.cu:7358-7385).  Scales and quaternions are read at
// slot src[i] (caller order, for the deformed shapes) or i (internal order, rest shapes).
__global__ void __launch_bounds__(kBlock) k_contact_pack(int n, const float* __restrict__ sc,
	const float* __restrict__ qt, const int* __restrict__ src, const float* __restrict__ opacity, float tau,
	float rcap, float4* __restrict__ shape, float* __restrict__ rmax)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int s = src ? src[i] : i;
	const float a = opacity[i];
	const float k = (a > tau && tau > 0.0f) ? sqrtf(2.0f * logf(a / tau)) : 0.0f;
	float e0 = k * sc[3 * s], e1 = k * sc[3 * s + 1], e2 = k * sc[3 * s + 2];
	if (rcap > 0.0f) { e0 = fminf(e0, rcap); e1 = fminf(e1, rcap); e2 = fminf(e2, rcap); }
	if (!(isfinite(e0) && isfinite(e1) && isfinite(e2))) e0 = e1 = e2 = 0.0f;
	float w = qt[4 * s], x = qt[4 * s + 1], y = qt[4 * s + 2], z = qt[4 * s + 3];
	const float qn = sqrtf(w * w + x * x + y * y + z * z);
	if (qn > 1e-20f) { w /= qn; x /= qn; y /= qn; z /= qn; }
	else { w = 1.0f; x = y = z = 0.0f; }
	// rotation whose columns are the Gaussian's local axes
	const float r00 = 1 - 2 * (y * y + z * z), r01 = 2 * (x * y - w * z), r02 = 2 * (x * z + w * y);
	const float r10 = 2 * (x * y + w * z), r11 = 1 - 2 * (x * x + z * z), r12 = 2 * (y * z - w * x);
	const float r20 = 2 * (x * z - w * y), r21 = 2 * (y * z + w * x), r22 = 1 - 2 * (x * x + y * y);
	const float l0 = e0 * e0, l1 = e1 * e1, l2 = e2 * e2;
	shape[2 * i] = make_float4(r00 * r00 * l0 + r01 * r01 * l1 + r02 * r02 * l2,
		r00 * r10 * l0 + r01 * r11 * l1 + r02 * r12 * l2,
		r00 * r20 * l0 + r01 * r21 * l1 + r02 * r22 * l2,
		r10 * r10 * l0 + r11 * r11 * l1 + r12 * r12 * l2);
	shape[2 * i + 1] = make_float4(r10 * r20 * l0 + r11 * r21 * l1 + r12 * r22 * l2,
		r20 * r20 * l0 + r21 * r21 * l1 + r22 * r22 * l2, 0.0f, 0.0f);
	rmax[i] = fmaxf(e0, fmaxf(e1, e2));
}

// ---------------------------------------------------------------------------
// predict (forward.cu:5954-5979); also clears the volume multipliers of the step
// (forward.cu:12058-12060) and, with ellipsoid ground contact on, refreshes each
// Gaussian's support radius along the ground normal (contactGroundRadiusKernel,
// forward.cu:7394-7399, run once per step at 12223-12227).  HBM: 16+16 B read, 16+16 B
// written per Gaussian (+32 B read, 4 B written with ground contact shapes).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void predict_row(int i, int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pos_curr, float4* __restrict__ pos_next, float4* __restrict__ vel,
	float* __restrict__ lam_vol, const float4* __restrict__ cshape, float* __restrict__ crg)
{
	if (i >= n) return;
	const float4 x4 = pos_curr[i];
	float4 v4 = vel[i];
	const float dt = P->dt;
	const float3 g = make_float3(P->gx, P->gy, P->gz);
	if (lam_vol) lam_vol[i] = 0.0f;
	if (crg) crg[i] = contact_support(cshape[2 * i], cshape[2 * i + 1], P->gn[0], P->gn[1], P->gn[2]);
	if (x4.w > 0.0f) {
		float3 v = add3(f3(v4), mul3(g, dt));
		const float3 p = add3(f3(x4), mul3(v, dt));
		pos_next[i] = make_float4(p.x, p.y, p.z, x4.w);
		vel[i] = make_float4(v.x, v.y, v.z, 0.0f);
	}
	else {
		pos_next[i] = x4;
		vel[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	}
}
__global__ void __launch_bounds__(kBlock) k_predict(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pos_curr, float4* __restrict__ pos_next, float4* __restrict__ vel,
	float* __restrict__ lam_vol, const float4* __restrict__ cshape, float* __restrict__ crg)
{
	predict_row(blockIdx.x * blockDim.x + threadIdx.x, n, P, pos_curr, pos_next, vel, lam_vol, cshape, crg);
}

// ---------------------------------------------------------------------------
// distance constraints, Jacobi (forward.cu:6484-6571).  One thread per Gaussian over
// its CSR row; the multiplier of each directed edge is owned by that thread, so it is
// updated in place (the reference ping-pongs two arrays; the value sequence per edge
// is the same).  The first iteration of a step reads no multiplier (they start at 0)
// and the last stores none (they are reset next step).
// ---------------------------------------------------------------------------
template <bool NC>
__device__ __forceinline__ void distance_row(int idx, int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, float4* __restrict__ pout, const int* __restrict__ off,
	const int* __restrict__ nbr, const float* __restrict__ ndist, const float* __restrict__ nstiff,
	float* __restrict__ lam, int read_lam, int write_lam)
{
	if (idx >= n) return;
	const float4 p4 = ldv<NC>(pin, idx);
	const float3 pi = f3(p4);
	const float ims = P->inv_mass_scale, ss = P->stiffness_scale, gc = P->dist_compliance;
	const float wi = p4.w * ims;
	float3 accum = make_float3(0.0f, 0.0f, 0.0f);
	int valid = 0;
	const float dt = P->dt;
	const float dt2 = fmaxf(dt * dt, 1e-8f);
	const int e0 = off[idx], e1 = off[idx + 1];
	// one edge of the row: its neighbour's position and its own multiplier, rest length
	// and stiffness already loaded
	auto edge_step = [&](int edge, float4 q4, float lambda, float rest, float stiff_e) {
		const float3 diff = sub3(pi, f3(q4));
		const float d = len3(diff);
		if (d < 1e-7f) return;
		const float C = d - rest;
		const float3 grad = mul3(diff, 1.0f / d);
		const float wj = q4.w * ims;
		const float stiff = fmaxf(stiff_e * ss, 1e-6f);
		const float alpha = gc / stiff;
		const float alpha_tilde = alpha / dt2;
		const float denom = (wi + wj) + alpha_tilde;
		if (denom < 1e-8f) return;
		const float dl = (-C - alpha_tilde * lambda) / denom;
		lambda += dl;
		if (write_lam) lam[edge] = lambda;
		if (wi > 0.0f) {
			accum = add3(accum, mul3(grad, wi * dl));
			valid++;
		}
	};
	// two edges per trip: their loads are in flight together; edges are applied in row
	// order, so the result is that of the one-at-a-time loop bit for bit
	int edge = e0;
	for (; edge + 1 < e1; edge += 2) {
		const int j0 = __ldg(nbr + edge), j1 = __ldg(nbr + edge + 1);
		const float l0 = read_lam ? lam[edge] : 0.0f, l1 = read_lam ? lam[edge + 1] : 0.0f;
		const bool ok0 = j0 >= 0 && j0 < n, ok1 = j1 >= 0 && j1 < n;
		float4 q0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), q1 = q0;
		if (ok0) q0 = ldv<NC>(pin, j0);
		if (ok1) q1 = ldv<NC>(pin, j1);
		const float r0 = __ldg(ndist + edge), r1 = __ldg(ndist + edge + 1);
		const float s0 = __ldg(nstiff + edge), s1 = __ldg(nstiff + edge + 1);
		if (ok0) edge_step(edge, q0, l0, r0, s0);
		if (ok1) edge_step(edge + 1, q1, l1, r1, s1);
	}
	if (edge < e1) {
		const int j = __ldg(nbr + edge);
		const float lambda = read_lam ? lam[edge] : 0.0f;
		if (j >= 0 && j < n) edge_step(edge, ldv<NC>(pin, j), lambda, __ldg(ndist + edge), __ldg(nstiff + edge));
	}
	float3 out = pi;
	if (wi > 0.0f && valid > 0) {
		const float3 avg = mul3(accum, 1.0f / float(valid));
		out = add3(pi, mul3(avg, P->under_relax));
	}
	pout[idx] = make_float4(out.x, out.y, out.z, p4.w);
}
__global__ void __launch_bounds__(kBlock) k_distance_jacobi(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, float4* __restrict__ pout, const int* __restrict__ off,
	const int* __restrict__ nbr, const float* __restrict__ ndist, const float* __restrict__ nstiff,
	float* __restrict__ lam, int read_lam, int write_lam)
{
	distance_row<true>(blockIdx.x * blockDim.x + threadIdx.x, n, P, pin, pout, off, nbr, ndist, nstiff, lam, read_lam,
		write_lam);
}
template <int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_distance_occ(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, float4* __restrict__ pout, const int* __restrict__ off,
	const int* __restrict__ nbr, const float* __restrict__ ndist, const float* __restrict__ nstiff,
	float* __restrict__ lam, int read_lam, int write_lam)
{
	distance_row<true>(blockIdx.x * blockDim.x + threadIdx.x, n, P, pin, pout, off, nbr, ndist, nstiff, lam, read_lam,
		write_lam);
}

// distance Gauss-Seidel, one colour: thread per undirected edge, in place
// (forward.cu:6576-6621)
__global__ void __launch_bounds__(kBlock) k_distance_gs(int begin, int count, int n, const StepParams* __restrict__ P,
	float4* __restrict__ pos, const int2* __restrict__ edge, const float* __restrict__ rest,
	const float* __restrict__ stiff, float* __restrict__ lam, int read_lam)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= count) return;
	const int e = begin + t;
	const int2 ij = edge[e];
	if (ij.x < 0 || ij.x >= n || ij.y < 0 || ij.y >= n) return;
	const float4 a = pos[ij.x], b = pos[ij.y];
	const float ims = P->inv_mass_scale;
	const float wi = a.w * ims, wj = b.w * ims;
	if (wi + wj <= 0.0f) return;
	const float3 pi = f3(a), pj = f3(b);
	const float3 diff = sub3(pi, pj);
	const float d = len3(diff);
	if (d < 1e-7f) return;
	const float dt = P->dt;
	const float dt2 = fmaxf(dt * dt, 1e-8f);
	const float s = fmaxf(stiff[e] * P->stiffness_scale, 1e-6f);
	const float alpha_tilde = (P->dist_compliance / s) / dt2;
	const float denom = (wi + wj) + alpha_tilde;
	if (denom < 1e-8f) return;
	const float C = d - rest[e];
	const float l = read_lam ? lam[e] : 0.0f;
	const float dl = (-C - alpha_tilde * l) / denom;
	lam[e] = l + dl;
	const float3 nn = mul3(diff, 1.0f / d);
	if (wi > 0.0f) { const float3 o = add3(pi, mul3(nn, wi * dl)); pos[ij.x] = make_float4(o.x, o.y, o.z, a.w); }
	if (wj > 0.0f) { const float3 o = sub3(pj, mul3(nn, wj * dl)); pos[ij.y] = make_float4(o.x, o.y, o.z, b.w); }
}

// ---------------------------------------------------------------------------
// volume: J and Sigma^-1 of one cluster covariance (forward.cu:8583-8620)
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool cluster_j_sinv(const M3& Scur, float det_rest, float& J, float& C, M3& Sinv)
{
	float s_cur, det_hat;
	if (!sigma_scale_det(Scur, s_cur, det_hat)) return false;
	const float det_cur = s_cur * s_cur * s_cur * det_hat;
	if (det_rest < 1e-30f) return false;
	J = sqrtf(det_cur / det_rest);
	if (!isfinite(J) || J <= 0.0f) return false;
	if (J > 3.0f || J < 0.333f) J = fminf(3.0f, fmaxf(0.333f, J));
	C = J - 1.0f;
	if (fabsf(C) < 1e-4f) return false;
	M3 Sreg = Scur;
	if (det_hat < 0.2f) {
		const float d = 0.06f * s_cur;
		Sreg.m[0][0] += d; Sreg.m[1][1] += d; Sreg.m[2][2] += d;
	}
	return inverse3x3_safe(Sreg, Sinv, 1e-20f);
}

// Cluster blackboard record, 36 bytes: one aligned 32-byte sector rec[2i], rec[2i + 1] =
// (M00, M11, M22, M01), (M02, M12, c.x, c.y) with M = coef Sinv, and c.z in the float
// array recz[i].  A record the gather must skip (the reference's coef == 0) has c.x =
// NaN.  The gather fetches the sector with one 256-bit load (ld.global.v8.f32, sm_100).
__device__ __forceinline__ int rec_a(int i) { return 2 * i; }
__device__ __forceinline__ int rec_b(int i) { return 2 * i + 1; }
// both halves of record i in one 256-bit load; NC: read-only path (records written by an
// earlier launch), else a coherent load (records written earlier in the same launch)
template <bool NC>
__device__ __forceinline__ void ld_rec(const float4* rec, int i, float4& a, float4& b)
{
	const float4* p = rec + 2 * (size_t)i;
	if (NC)
		asm volatile("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
			: "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w) : "l"(p));
	else
		asm volatile("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
			: "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w) : "l"(p) : "memory");
}
__device__ __forceinline__ void rec_invalidate(float4* rec, int idx) { rec[rec_b(idx)].z = __int_as_float(0x7fc00000); }
__device__ __forceinline__ void store_record(float4* rec, float* recz, int idx, float3 c, float coef, const M3& S)
{
	if (coef == 0.0f) { rec_invalidate(rec, idx); return; }
	rec[rec_a(idx)] = make_float4(coef * S.m[0][0], coef * S.m[1][1], coef * S.m[2][2], coef * S.m[1][0]);
	rec[rec_b(idx)] = make_float4(coef * S.m[2][0], coef * S.m[2][1], c.x, c.y);
	recz[idx] = c.z;
}

// Kernel A on groups of S lanes per cluster (32/S clusters per warp).  Lane L of a group
// owns members L, L+S, ...; their positions stay in registers (VC slots) across the
// centroid, covariance and denominator passes, and butterfly sums inside the group give
// every lane the totals.  S = 32 is the reference's warp kernel with its exact summation
// order (forward.cu:8702-8863); smaller S runs the same operations with the per-cluster
// serial 3x3 work (J, Sigma^-1) shared by fewer lanes, i.e. more clusters per warp
// instruction.  No lane leaves before the last shuffle, so groups may diverge freely.
// Reads per cluster: m member indices (coalesced runs of S) + m gathered positions.
template <int S>
__device__ __forceinline__ float group_sum(float v)
{
#pragma unroll
	for (int o = S / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

template <int S, int VC>
__global__ void __launch_bounds__(kBlock) k_volume_solve_group(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, const int* __restrict__ voff, const int* __restrict__ vidx,
	const float* __restrict__ det_rest, const int* __restrict__ mat_type, float* __restrict__ lam_vol,
	float4* __restrict__ rec, float* __restrict__ recz, int read_lam)
{
	const int sl = threadIdx.x & (S - 1);
	const int idx = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) / S);
	const bool in_range = idx < n;
	bool valid = in_range && mat_type[idx] == 0;
	int off = 0, cnt = 0;
	float4 p4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	if (valid) {
		off = voff[idx];
		cnt = voff[idx + 1] - off;
		p4 = ld4(pin, idx);
	}
	const float3 pi = f3(p4);
	float3 cache[VC];
	float cw[VC];
	int nc = 0, ucnt = 0;
	float3 psum = make_float3(0.0f, 0.0f, 0.0f);
	for (int k = sl; k < cnt; k += S) {
		const int j = __ldg(vidx + off + k);
		if (j < 0 || j >= n) continue;
		const float4 q = ld4(pin, j);
		psum = add3(psum, f3(q));
		++ucnt;
#pragma unroll
		for (int t = 0; t < VC; ++t)
			if (t == nc) { cache[t] = f3(q); cw[t] = q.w; }
		if (nc < VC) ++nc;
	}
	const float sx = group_sum<S>(psum.x), sy = group_sum<S>(psum.y), sz = group_sum<S>(psum.z);
	const int used = (int)(group_sum<S>((float)ucnt) + 0.5f);
	valid = valid && used >= 3;
	const float inv_n = 1.0f / (float)(used + 1);
	const float3 c = make_float3((sx + pi.x) * inv_n, (sy + pi.y) * inv_n, (sz + pi.z) * inv_n);
	float a00 = 0.f, a11 = 0.f, a22 = 0.f, a01 = 0.f, a02 = 0.f, a12 = 0.f;
#pragma unroll
	for (int t = 0; t < VC; ++t) {
		if (t < nc) {
			const float dx = cache[t].x - c.x, dy = cache[t].y - c.y, dz = cache[t].z - c.z;
			a00 += dx * dx; a11 += dy * dy; a22 += dz * dz;
			a01 += dx * dy; a02 += dx * dz; a12 += dy * dz;
		}
	}
	if (ucnt > nc) {
		int seen = 0;
		for (int k = sl; k < cnt; k += S) {
			const int j = __ldg(vidx + off + k);
			if (j < 0 || j >= n) continue;
			if (seen++ < nc) continue;
			const float3 q = f3(ld4(pin, j));
			const float dx = q.x - c.x, dy = q.y - c.y, dz = q.z - c.z;
			a00 += dx * dx; a11 += dy * dy; a22 += dz * dz;
			a01 += dx * dy; a02 += dx * dz; a12 += dy * dz;
		}
	}
	if (sl == 0) {
		const float dx = pi.x - c.x, dy = pi.y - c.y, dz = pi.z - c.z;
		a00 += dx * dx; a11 += dy * dy; a22 += dz * dz;
		a01 += dx * dy; a02 += dx * dz; a12 += dy * dz;
	}
	M3 Sm;
	Sm.m[0][0] = group_sum<S>(a00) * inv_n;
	Sm.m[1][1] = group_sum<S>(a11) * inv_n;
	Sm.m[2][2] = group_sum<S>(a22) * inv_n;
	const float s01 = group_sum<S>(a01) * inv_n, s02 = group_sum<S>(a02) * inv_n, s12 = group_sum<S>(a12) * inv_n;
	Sm.m[0][1] = Sm.m[1][0] = s01;
	Sm.m[0][2] = Sm.m[2][0] = s02;
	Sm.m[1][2] = Sm.m[2][1] = s12;
	float J = 1.0f, C = 0.0f;
	M3 Sinv;
	m3_zero(Sinv);
	if (valid) valid = cluster_j_sinv(Sm, __ldg(det_rest + idx), J, C, Sinv);
	const float gs = J * inv_n;
	const float ims = P->inv_mass_scale;
	float dsum = 0.0f;
	if (valid) {
#pragma unroll
		for (int t = 0; t < VC; ++t) {
			if (t < nc) {
				const float3 g = mul3(m3_mulv(Sinv, make_float3(cache[t].x - c.x, cache[t].y - c.y, cache[t].z - c.z)), gs);
				dsum += (cw[t] * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
			}
		}
		if (ucnt > nc) {
			int seen = 0;
			for (int k = sl; k < cnt; k += S) {
				const int j = __ldg(vidx + off + k);
				if (j < 0 || j >= n) continue;
				if (seen++ < nc) continue;
				const float4 q = ld4(pin, j);
				const float3 g = mul3(m3_mulv(Sinv, make_float3(q.x - c.x, q.y - c.y, q.z - c.z)), gs);
				dsum += (q.w * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
			}
		}
		if (sl == 0) {
			const float3 g = mul3(m3_mulv(Sinv, make_float3(pi.x - c.x, pi.y - c.y, pi.z - c.z)), gs);
			dsum += (p4.w * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
		}
	}
	const float denom = group_sum<S>(dsum);
	if (sl != 0 || !in_range) return;
	if (!valid) { rec_invalidate(rec, idx); return; }
	const float dt = P->dt;
	const float dt2 = fmaxf(dt * dt, 1e-8f);
	const float alpha_t = P->vol_compliance / dt2;
	const float den = denom + alpha_t;
	if (!(den > 1e-12f)) { rec_invalidate(rec, idx); return; }
	const float lam = read_lam ? lam_vol[idx] : 0.0f;
	const float dl = (-C - alpha_t * lam) / den;
	if (!isfinite(dl)) { rec_invalidate(rec, idx); return; }
	lam_vol[idx] = lam + dl;
	store_record(rec, recz, idx, c, dl * gs, Sinv);
}

// Kernel A with static register slots: lane sl of an S-lane group owns members
// sl + t*S (t < NS) in fixed registers (index, and the position when CP), so the three
// passes over a cluster need no dynamic indexing; members past S*NS are streamed from
// memory in each pass.  Same per-lane order and arithmetic as k_volume_solve_group.
template <int S, int NS, bool CP>
__global__ void __launch_bounds__(kBlock) k_volume_solve_slots(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, const int* __restrict__ voff, const int* __restrict__ vidx,
	const float* __restrict__ det_rest, const int* __restrict__ mat_type, float* __restrict__ lam_vol,
	float4* __restrict__ rec, float* __restrict__ recz, int read_lam)
{
	const int sl = threadIdx.x & (S - 1);
	const int idx = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) / S);
	const bool in_range = idx < n;
	bool valid = in_range && mat_type[idx] == 0;
	int off = 0, cnt = 0;
	float4 p4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	if (valid) {
		off = voff[idx];
		cnt = voff[idx + 1] - off;
		p4 = ld4(pin, idx);
	}
	const float3 pi = f3(p4);
	int jj[NS];
	float4 qq[CP ? NS : 1];
	int ucnt = 0;
	float3 psum = make_float3(0.0f, 0.0f, 0.0f);
#pragma unroll
	for (int t = 0; t < NS; ++t) {
		const int k = sl + t * S;
		int j = -1;
		if (k < cnt) {
			j = __ldg(vidx + off + k);
			if (j >= n) j = -1;
		}
		jj[t] = j;
	}
#pragma unroll
	for (int t = 0; t < NS; ++t) {
		if (jj[t] >= 0) {
			const float4 q = ld4(pin, jj[t]);
			if (CP) qq[t] = q;
			psum = add3(psum, f3(q));
			++ucnt;
		}
	}
	for (int k = sl + NS * S; k < cnt; k += S) {
		const int j = __ldg(vidx + off + k);
		if (j < 0 || j >= n) continue;
		psum = add3(psum, f3(ld4(pin, j)));
		++ucnt;
	}
	const float sx = group_sum<S>(psum.x), sy = group_sum<S>(psum.y), sz = group_sum<S>(psum.z);
	const int used = (int)(group_sum<S>((float)ucnt) + 0.5f);
	valid = valid && used >= 3;
	const float inv_n = 1.0f / (float)(used + 1);
	const float3 c = make_float3((sx + pi.x) * inv_n, (sy + pi.y) * inv_n, (sz + pi.z) * inv_n);
	float a00 = 0.f, a11 = 0.f, a22 = 0.f, a01 = 0.f, a02 = 0.f, a12 = 0.f;
#pragma unroll
	for (int t = 0; t < NS; ++t) {
		if (jj[t] >= 0) {
			const float4 q = CP ? qq[t] : ld4(pin, jj[t]);
			const float dx = q.x - c.x, dy = q.y - c.y, dz = q.z - c.z;
			a00 += dx * dx; a11 += dy * dy; a22 += dz * dz;
			a01 += dx * dy; a02 += dx * dz; a12 += dy * dz;
		}
	}
	for (int k = sl + NS * S; k < cnt; k += S) {
		const int j = __ldg(vidx + off + k);
		if (j < 0 || j >= n) continue;
		const float3 q = f3(ld4(pin, j));
		const float dx = q.x - c.x, dy = q.y - c.y, dz = q.z - c.z;
		a00 += dx * dx; a11 += dy * dy; a22 += dz * dz;
		a01 += dx * dy; a02 += dx * dz; a12 += dy * dz;
	}
	if (sl == 0) {
		const float dx = pi.x - c.x, dy = pi.y - c.y, dz = pi.z - c.z;
		a00 += dx * dx; a11 += dy * dy; a22 += dz * dz;
		a01 += dx * dy; a02 += dx * dz; a12 += dy * dz;
	}
	M3 Sm;
	Sm.m[0][0] = group_sum<S>(a00) * inv_n;
	Sm.m[1][1] = group_sum<S>(a11) * inv_n;
	Sm.m[2][2] = group_sum<S>(a22) * inv_n;
	const float s01 = group_sum<S>(a01) * inv_n, s02 = group_sum<S>(a02) * inv_n, s12 = group_sum<S>(a12) * inv_n;
	Sm.m[0][1] = Sm.m[1][0] = s01;
	Sm.m[0][2] = Sm.m[2][0] = s02;
	Sm.m[1][2] = Sm.m[2][1] = s12;
	float J = 1.0f, C = 0.0f;
	M3 Sinv;
	m3_zero(Sinv);
	if (valid) valid = cluster_j_sinv(Sm, __ldg(det_rest + idx), J, C, Sinv);
	const float gs = J * inv_n;
	const float ims = P->inv_mass_scale;
	float dsum = 0.0f;
	if (valid) {
#pragma unroll
		for (int t = 0; t < NS; ++t) {
			if (jj[t] >= 0) {
				const float4 q = CP ? qq[t] : ld4(pin, jj[t]);
				const float3 g = mul3(m3_mulv(Sinv, make_float3(q.x - c.x, q.y - c.y, q.z - c.z)), gs);
				dsum += (q.w * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
			}
		}
		for (int k = sl + NS * S; k < cnt; k += S) {
			const int j = __ldg(vidx + off + k);
			if (j < 0 || j >= n) continue;
			const float4 q = ld4(pin, j);
			const float3 g = mul3(m3_mulv(Sinv, make_float3(q.x - c.x, q.y - c.y, q.z - c.z)), gs);
			dsum += (q.w * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
		}
		if (sl == 0) {
			const float3 g = mul3(m3_mulv(Sinv, make_float3(pi.x - c.x, pi.y - c.y, pi.z - c.z)), gs);
			dsum += (p4.w * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
		}
	}
	const float denom = group_sum<S>(dsum);
	if (sl != 0 || !in_range) return;
	if (!valid) { rec_invalidate(rec, idx); return; }
	const float dt = P->dt;
	const float dt2 = fmaxf(dt * dt, 1e-8f);
	const float alpha_t = P->vol_compliance / dt2;
	const float den = denom + alpha_t;
	if (!(den > 1e-12f)) { rec_invalidate(rec, idx); return; }
	const float lam = read_lam ? lam_vol[idx] : 0.0f;
	const float dl = (-C - alpha_t * lam) / den;
	if (!isfinite(dl)) { rec_invalidate(rec, idx); return; }
	lam_vol[idx] = lam + dl;
	store_record(rec, recz, idx, c, dl * gs, Sinv);
}

// Kernel A with the members' positions staged in shared memory: pass 1 gathers each
// lane's NS members once (L2/L1) and parks them in a per-thread column of shared memory
// (slot t of thread x at [t][x], so a warp's accesses are conflict-free); the covariance
// and denominator passes read them back from there instead of re-gathering.  Same
// per-lane order and arithmetic as k_volume_solve_slots.  Block size must be kSmemBlock.
constexpr int kSmemBlock = 128;
template <int S, int NS>
__global__ void __launch_bounds__(kSmemBlock) k_volume_solve_smem(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, const int* __restrict__ voff, const int* __restrict__ vidx,
	const float* __restrict__ det_rest, const int* __restrict__ mat_type, float* __restrict__ lam_vol,
	float4* __restrict__ rec, float* __restrict__ recz, int read_lam)
{
	__shared__ float4 stage[NS][kSmemBlock];
	const int tx = threadIdx.x;
	const int sl = tx & (S - 1);
	const int idx = (int)(((long long)blockIdx.x * kSmemBlock + tx) / S);
	const bool in_range = idx < n;
	bool valid = in_range && mat_type[idx] == 0;
	int off = 0, cnt = 0;
	float4 p4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	if (valid) {
		off = voff[idx];
		cnt = voff[idx + 1] - off;
		p4 = ld4(pin, idx);
	}
	const float3 pi = f3(p4);
	unsigned int live = 0u;   // bit t: slot t holds a member
	int ucnt = 0;
	float3 psum = make_float3(0.0f, 0.0f, 0.0f);
	{
		int jj[NS];
#pragma unroll
		for (int t = 0; t < NS; ++t) {
			const int k = sl + t * S;
			int j = -1;
			if (k < cnt) {
				j = __ldg(vidx + off + k);
				if (j >= n) j = -1;
			}
			jj[t] = j;
		}
#pragma unroll
		for (int t = 0; t < NS; ++t) {
			if (jj[t] >= 0) {
				const float4 q = ld4(pin, jj[t]);
				stage[t][tx] = q;
				live |= 1u << t;
				psum = add3(psum, f3(q));
				++ucnt;
			}
		}
	}
	for (int k = sl + NS * S; k < cnt; k += S) {
		const int j = __ldg(vidx + off + k);
		if (j < 0 || j >= n) continue;
		psum = add3(psum, f3(ld4(pin, j)));
		++ucnt;
	}
	const float sx = group_sum<S>(psum.x), sy = group_sum<S>(psum.y), sz = group_sum<S>(psum.z);
	const int used = (int)(group_sum<S>((float)ucnt) + 0.5f);
	valid = valid && used >= 3;
	const float inv_n = 1.0f / (float)(used + 1);
	const float3 c = make_float3((sx + pi.x) * inv_n, (sy + pi.y) * inv_n, (sz + pi.z) * inv_n);
	float a00 = 0.f, a11 = 0.f, a22 = 0.f, a01 = 0.f, a02 = 0.f, a12 = 0.f;
#pragma unroll
	for (int t = 0; t < NS; ++t) {
		if (live & (1u << t)) {
			const float4 q = stage[t][tx];
			const float dx = q.x - c.x, dy = q.y - c.y, dz = q.z - c.z;
			a00 += dx * dx; a11 += dy * dy; a22 += dz * dz;
			a01 += dx * dy; a02 += dx * dz; a12 += dy * dz;
		}
	}
	for (int k = sl + NS * S; k < cnt; k += S) {
		const int j = __ldg(vidx + off + k);
		if (j < 0 || j >= n) continue;
		const float3 q = f3(ld4(pin, j));
		const float dx = q.x - c.x, dy = q.y - c.y, dz = q.z - c.z;
		a00 += dx * dx; a11 += dy * dy; a22 += dz * dz;
		a01 += dx * dy; a02 += dx * dz; a12 += dy * dz;
	}
	if (sl == 0) {
		const float dx = pi.x - c.x, dy = pi.y - c.y, dz = pi.z - c.z;
		a00 += dx * dx; a11 += dy * dy; a22 += dz * dz;
		a01 += dx * dy; a02 += dx * dz; a12 += dy * dz;
	}
	M3 Sm;
	Sm.m[0][0] = group_sum<S>(a00) * inv_n;
	Sm.m[1][1] = group_sum<S>(a11) * inv_n;
	Sm.m[2][2] = group_sum<S>(a22) * inv_n;
	const float s01 = group_sum<S>(a01) * inv_n, s02 = group_sum<S>(a02) * inv_n, s12 = group_sum<S>(a12) * inv_n;
	Sm.m[0][1] = Sm.m[1][0] = s01;
	Sm.m[0][2] = Sm.m[2][0] = s02;
	Sm.m[1][2] = Sm.m[2][1] = s12;
	float J = 1.0f, C = 0.0f;
	M3 Sinv;
	m3_zero(Sinv);
	if (valid) valid = cluster_j_sinv(Sm, __ldg(det_rest + idx), J, C, Sinv);
	const float gs = J * inv_n;
	const float ims = P->inv_mass_scale;
	float dsum = 0.0f;
	if (valid) {
#pragma unroll
		for (int t = 0; t < NS; ++t) {
			if (live & (1u << t)) {
				const float4 q = stage[t][tx];
				const float3 g = mul3(m3_mulv(Sinv, make_float3(q.x - c.x, q.y - c.y, q.z - c.z)), gs);
				dsum += (q.w * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
			}
		}
		for (int k = sl + NS * S; k < cnt; k += S) {
			const int j = __ldg(vidx + off + k);
			if (j < 0 || j >= n) continue;
			const float4 q = ld4(pin, j);
			const float3 g = mul3(m3_mulv(Sinv, make_float3(q.x - c.x, q.y - c.y, q.z - c.z)), gs);
			dsum += (q.w * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
		}
		if (sl == 0) {
			const float3 g = mul3(m3_mulv(Sinv, make_float3(pi.x - c.x, pi.y - c.y, pi.z - c.z)), gs);
			dsum += (p4.w * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
		}
	}
	const float denom = group_sum<S>(dsum);
	if (sl != 0 || !in_range) return;
	if (!valid) { rec_invalidate(rec, idx); return; }
	const float dt = P->dt;
	const float dt2 = fmaxf(dt * dt, 1e-8f);
	const float alpha_t = P->vol_compliance / dt2;
	const float den = denom + alpha_t;
	if (!(den > 1e-12f)) { rec_invalidate(rec, idx); return; }
	const float lam = read_lam ? lam_vol[idx] : 0.0f;
	const float dl = (-C - alpha_t * lam) / den;
	if (!isfinite(dl)) { rec_invalidate(rec, idx); return; }
	lam_vol[idx] = lam + dl;
	store_record(rec, recz, idx, c, dl * gs, Sinv);
}

// Kernel A in one pass over the members (S lanes per cluster, members L, L+S, ... of
// the Morton-sorted list on lane L, two in flight per trip): each lane accumulates,
// relative to the leader's position, the count, first and second moments of its
// members and the same moments weighted by inverse mass.  The centred covariance
//   Sigma = (1 / (m+1)) sum (q - c)(q - c)^T = sum d d^T / (m+1) - c' c'^T
// (d = q - p_leader, c' = c - p_leader, the leader's d = 0) and the denominator
//   sum w |g Sinv (q - c)|^2 = g^2 tr(Sinv^2 W),  W = sum w (d - c')(d - c')^T
// follow from them, so the member positions are read once and nothing is staged.
// Members lie within a few graph spacings of their leader, which keeps the
// cancellation in the moment form small; the result equals the two-pass form
// (forward.cu:8531-8664) to FP32 rounding.  The reference has the same leader-relative
// moments in its optional one-pass warp kernel (forward.cu:8864-9033, warp mode 3).
template <int S, bool NC>
__device__ __forceinline__ void solve_onepass_lane(long long gtid, int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, const int* __restrict__ voff, const int* __restrict__ vidx,
	const float* __restrict__ det_rest, const int* __restrict__ mat_type, float* __restrict__ lam_vol,
	float4* __restrict__ rec, float* __restrict__ recz, int read_lam)
{
	const int sl = (int)(gtid & (S - 1));
	const int idx = (int)(gtid / S);
	const bool in_range = idx < n;
	bool valid = in_range && mat_type[idx] == 0;
	int off = 0, cnt = 0;
	float4 p4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	if (valid) {
		off = voff[idx];
		cnt = voff[idx + 1] - off;
		p4 = ldv<NC>(pin, idx);
	}
	const float3 pi = f3(p4);
	const float ims = P->inv_mass_scale;
	// m[0..9]: count, d, d d^T (xx yy zz xy xz yz); m[10..19]: the same weighted by w.
	// The weighted sums are formed in a second pass over the members only when their
	// inverse masses differ; otherwise they are w times the plain ones
	float m[20];
#pragma unroll
	for (int t = 0; t < 20; ++t) m[t] = 0.0f;
	float wmin = INFINITY, wmax = -INFINITY;
	auto add = [&](float4 q) {
		const float dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z, w = q.w * ims;
		m[0] += 1.0f; m[1] += dx; m[2] += dy; m[3] += dz;
		m[4] += dx * dx; m[5] += dy * dy; m[6] += dz * dz; m[7] += dx * dy; m[8] += dx * dz; m[9] += dy * dz;
		wmin = fminf(wmin, w); wmax = fmaxf(wmax, w);
	};
	auto add_w = [&](float4 q) {
		const float dx = q.x - pi.x, dy = q.y - pi.y, dz = q.z - pi.z, w = q.w * ims;
		m[10] += w; m[11] += w * dx; m[12] += w * dy; m[13] += w * dz;
		m[14] += w * dx * dx; m[15] += w * dy * dy; m[16] += w * dz * dz;
		m[17] += w * dx * dy; m[18] += w * dx * dz; m[19] += w * dy * dz;
	};
	int k = sl;
	for (; k + S < cnt; k += 2 * S) {
		const int j0 = __ldg(vidx + off + k), j1 = __ldg(vidx + off + k + S);
		const bool ok0 = j0 >= 0 && j0 < n, ok1 = j1 >= 0 && j1 < n;
		float4 q0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), q1 = q0;
		if (ok0) q0 = ldv<NC>(pin, j0);
		if (ok1) q1 = ldv<NC>(pin, j1);
		if (ok0) add(q0);
		if (ok1) add(q1);
	}
	if (k < cnt) {
		const int j = __ldg(vidx + off + k);
		if (j >= 0 && j < n) add(ldv<NC>(pin, j));
	}
#pragma unroll
	for (int t = 0; t < 10; ++t) m[t] = group_sum<S>(m[t]);
#pragma unroll
	for (int o = 1; o < S; o <<= 1) {
		wmin = fminf(wmin, __shfl_xor_sync(0xffffffffu, wmin, o, S));
		wmax = fmaxf(wmax, __shfl_xor_sync(0xffffffffu, wmax, o, S));
	}
	const bool mixed = wmin < wmax;   // warp-uniform second pass (full-warp shuffles)
	if (__any_sync(0xffffffffu, mixed)) {
		if (mixed)
			for (int k2 = sl; k2 < cnt; k2 += S) {
				const int j = __ldg(vidx + off + k2);
				if (j >= 0 && j < n) add_w(ldv<NC>(pin, j));
			}
#pragma unroll
		for (int t = 10; t < 20; ++t) m[t] = group_sum<S>(m[t]);
	}
	if (!mixed) {   // one inverse mass over the members (or no member)
		const float w0 = wmin <= wmax ? wmin : 0.0f;
#pragma unroll
		for (int t = 0; t < 10; ++t) m[10 + t] = w0 * m[t];
	}
	const int used = (int)(m[0] + 0.5f);
	valid = valid && used >= 3;
	const float inv_n = 1.0f / (float)(used + 1);
	const float cx = m[1] * inv_n, cy = m[2] * inv_n, cz = m[3] * inv_n;   // c - p_leader
	const float3 c = make_float3(pi.x + cx, pi.y + cy, pi.z + cz);
	M3 Sm;
	Sm.m[0][0] = m[4] * inv_n - cx * cx;
	Sm.m[1][1] = m[5] * inv_n - cy * cy;
	Sm.m[2][2] = m[6] * inv_n - cz * cz;
	Sm.m[0][1] = Sm.m[1][0] = m[7] * inv_n - cx * cy;
	Sm.m[0][2] = Sm.m[2][0] = m[8] * inv_n - cx * cz;
	Sm.m[1][2] = Sm.m[2][1] = m[9] * inv_n - cy * cz;
	if (sl != 0 || !in_range) return;
	float J = 1.0f, C = 0.0f;
	M3 Sinv;
	m3_zero(Sinv);
	if (valid) valid = cluster_j_sinv(Sm, __ldg(det_rest + idx), J, C, Sinv);
	if (!valid) { rec_invalidate(rec, idx); return; }
	const float gs = J * inv_n;
	// W over members and leader (weight w_leader, d = 0)
	const float wl = p4.w * ims;
	const float ws = m[10] + wl;
	float W[3][3];
	const float wd[3] = { m[11], m[12], m[13] }, cc[3] = { cx, cy, cz };
	const float wdd[3][3] = { { m[14], m[17], m[18] }, { m[17], m[15], m[19] }, { m[18], m[19], m[16] } };
#pragma unroll
	for (int a = 0; a < 3; ++a)
#pragma unroll
		for (int b = 0; b < 3; ++b) W[a][b] = wdd[a][b] - cc[a] * wd[b] - wd[a] * cc[b] + ws * cc[a] * cc[b];
	// tr(Sinv^2 W) = sum_ab (Sinv^2)_ab W_ab
	float dsum = 0.0f;
#pragma unroll
	for (int a = 0; a < 3; ++a)
#pragma unroll
		for (int b = 0; b < 3; ++b) {
			const float s2 = Sinv.m[a][0] * Sinv.m[0][b] + Sinv.m[a][1] * Sinv.m[1][b] + Sinv.m[a][2] * Sinv.m[2][b];
			dsum += s2 * W[a][b];
		}
	const float denom = gs * gs * dsum;
	const float dt = P->dt;
	const float dt2 = fmaxf(dt * dt, 1e-8f);
	const float alpha_t = P->vol_compliance / dt2;
	const float den = denom + alpha_t;
	if (!(den > 1e-12f)) { rec_invalidate(rec, idx); return; }
	const float lam = read_lam ? lam_vol[idx] : 0.0f;
	const float dl = (-C - alpha_t * lam) / den;
	if (!isfinite(dl)) { rec_invalidate(rec, idx); return; }
	lam_vol[idx] = lam + dl;
	store_record(rec, recz, idx, c, dl * gs, Sinv);
}
template <int S>
__global__ void __launch_bounds__(kBlock) k_volume_solve_onepass(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, const int* __restrict__ voff, const int* __restrict__ vidx,
	const float* __restrict__ det_rest, const int* __restrict__ mat_type, float* __restrict__ lam_vol,
	float4* __restrict__ rec, float* __restrict__ recz, int read_lam)
{
	solve_onepass_lane<S, true>((long long)blockIdx.x * blockDim.x + threadIdx.x, n, P, pin,
		voff, vidx, det_rest, mat_type, lam_vol, rec, recz, read_lam);
}
template <int S, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_volume_solve_occ(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, const int* __restrict__ voff, const int* __restrict__ vidx,
	const float* __restrict__ det_rest, const int* __restrict__ mat_type, float* __restrict__ lam_vol,
	float4* __restrict__ rec, float* __restrict__ recz, int read_lam)
{
	solve_onepass_lane<S, true>((long long)blockIdx.x * blockDim.x + threadIdx.x, n, P, pin,
		voff, vidx, det_rest, mat_type, lam_vol, rec, recz, read_lam);
}

// Kernel A, one thread per cluster (forward.cu:8531-8664): sequential sums, leader first.
__global__ void __launch_bounds__(kBlock) k_volume_solve_thread(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, const int* __restrict__ voff, const int* __restrict__ vidx,
	const float* __restrict__ det_rest, const int* __restrict__ mat_type, float* __restrict__ lam_vol,
	float4* __restrict__ rec, float* __restrict__ recz, int read_lam)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= n) return;
	rec_invalidate(rec, idx);
	if (mat_type[idx] != 0) return;
	const float4 p4 = ld4(pin, idx);
	const float3 pi = f3(p4);
	const int off = voff[idx], cnt = voff[idx + 1] - off;
	float3 c = pi;
	int used = 0;
	for (int k = 0; k < cnt; ++k) {
		const int j = __ldg(vidx + off + k);
		if (j < 0 || j >= n) continue;
		c = add3(c, f3(ld4(pin, j)));
		++used;
	}
	if (used < 3) return;
	const float inv_n = 1.0f / (float)(used + 1);
	c = mul3(c, inv_n);
	M3 S;
	m3_zero(S);
	{
		const float3 d = sub3(pi, c);
		m3_add_outer(S, d, d);
	}
	for (int k = 0; k < cnt; ++k) {
		const int j = __ldg(vidx + off + k);
		if (j < 0 || j >= n) continue;
		const float3 d = sub3(f3(ld4(pin, j)), c);
		m3_add_outer(S, d, d);
	}
#pragma unroll
	for (int cc = 0; cc < 3; ++cc)
#pragma unroll
		for (int r = 0; r < 3; ++r) S.m[cc][r] *= inv_n;
	float J, C;
	M3 Sinv;
	if (!cluster_j_sinv(S, __ldg(det_rest + idx), J, C, Sinv)) return;
	const float gs = J * inv_n;
	const float ims = P->inv_mass_scale;
	float denom = 0.0f;
	{
		const float3 g = mul3(m3_mulv(Sinv, sub3(pi, c)), gs);
		denom += (p4.w * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
	}
	for (int k = 0; k < cnt; ++k) {
		const int j = __ldg(vidx + off + k);
		if (j < 0 || j >= n) continue;
		const float4 q = ld4(pin, j);
		const float3 g = mul3(m3_mulv(Sinv, sub3(f3(q), c)), gs);
		denom += (q.w * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
	}
	const float dt = P->dt;
	const float dt2 = fmaxf(dt * dt, 1e-8f);
	const float alpha_t = P->vol_compliance / dt2;
	const float den = denom + alpha_t;
	if (!(den > 1e-12f)) return;
	const float lam = read_lam ? lam_vol[idx] : 0.0f;
	const float dl = (-C - alpha_t * lam) / den;
	if (!isfinite(dl)) return;
	lam_vol[idx] = lam + dl;
	store_record(rec, recz, idx, c, dl * gs, Sinv);
}

// one blackboard record (already loaded) applied to a node (forward.cu:9212-9222):
// dp = w coef Sinv (p - c), skipped where the cluster gave no record
__device__ __forceinline__ bool gather_rec(float4 r0, float4 r1, float cz, float3 pi, float wi, float3& dp)
{
	if (!isfinite(r1.z)) return false;
	M3 M;
	M.m[0][0] = r0.x; M.m[1][1] = r0.y; M.m[2][2] = r0.z;
	M.m[0][1] = M.m[1][0] = r0.w;
	M.m[0][2] = M.m[2][0] = r1.x;
	M.m[1][2] = M.m[2][1] = r1.y;
	const float3 d = sub3(pi, make_float3(r1.z, r1.w, cz));
	const float3 g = m3_mulv(M, d);
	dp = make_float3(g.x * wi, g.y * wi, g.z * wi);
	return fin3(dp);
}

__device__ __forceinline__ bool gather_one(const float4* __restrict__ rec, const float* __restrict__ recz, int i, float3 pi, float wi,
	float3& dp)
{
	return gather_rec(__ldg(rec + rec_a(i)), __ldg(rec + rec_b(i)), __ldg(recz + i), pi, wi, dp);
}

__device__ __forceinline__ float3 gather_finish(float3 pi, float3 avg, float rl, float under_relax)
{
	if (rl > 1e-12f) {
		const float max_step = 0.25f * rl;
		const float len = len3(avg);
		if (len > max_step && len > 1e-20f) avg = mul3(avg, max_step / len);
	}
	return add3(pi, mul3(avg, under_relax));
}

// Kernel B on groups of S lanes per node (forward.cu:9262-9323 with S = 32): mean over
// the clusters that contain the node, step clamp 0.25 restLen, under-relaxation.  Reads
// per node: h reverse indices + h gathered 36-byte records (L2-resident).
template <int S, bool NC>
__device__ __forceinline__ void gather_group_lane(long long gtid, int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, float4* __restrict__ pout, const int* __restrict__ roff,
	const int* __restrict__ ridx, const float4* __restrict__ rec, const float* __restrict__ recz,
	const float* __restrict__ rest_len)
{
	const int sl = (int)(gtid & (S - 1));
	const int idx = (int)(gtid / S);
	const bool in_range = idx < n;
	float4 p4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	int off = 0, cnt = 0;
	float wi = 0.0f;
	if (in_range) {
		p4 = ldv<NC>(pin, idx);
		wi = p4.w * P->inv_mass_scale;
		if (wi > 0.0f) {
			off = roff[idx];
			cnt = roff[idx + 1] - off;
		}
	}
	const float3 pi = f3(p4);
	float3 sum = make_float3(0.0f, 0.0f, 0.0f);
	int received = 0;
	// two records per trip: both index loads, then all six record loads, are in flight
	// together (the loop is latency bound); records are applied in list order, as in
	// the one-at-a-time loop, so the sum is the same bit for bit
	int k = sl;
	for (; k + S < cnt; k += 2 * S) {
		const int i0 = __ldg(ridx + off + k), i1 = __ldg(ridx + off + k + S);
		const bool ok0 = i0 >= 0 && i0 < n, ok1 = i1 >= 0 && i1 < n;
		float4 a0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), b0 = a0, a1 = a0, b1 = a0;
		float z0 = 0.0f, z1 = 0.0f;
		const float* cz = recz;
		if (ok0) { ld_rec<NC>(rec, i0, a0, b0); z0 = ldv<NC>(cz, i0); }
		if (ok1) { ld_rec<NC>(rec, i1, a1, b1); z1 = ldv<NC>(cz, i1); }
		float3 dp;
		if (ok0 && gather_rec(a0, b0, z0, pi, wi, dp)) { sum = add3(sum, dp); ++received; }
		if (ok1 && gather_rec(a1, b1, z1, pi, wi, dp)) { sum = add3(sum, dp); ++received; }
	}
	if (k < cnt) {
		const int i = __ldg(ridx + off + k);
		float3 dp;
		float4 a = make_float4(0.0f, 0.0f, 0.0f, 0.0f), b = a;
		if (i >= 0 && i < n) ld_rec<NC>(rec, i, a, b);
		if (i >= 0 && i < n && gather_rec(a, b, ldv<NC>(recz, i), pi, wi, dp)) {
			sum = add3(sum, dp);
			++received;
		}
	}
	const float sx = group_sum<S>(sum.x), sy = group_sum<S>(sum.y), sz = group_sum<S>(sum.z);
	const int rc = (int)(group_sum<S>((float)received) + 0.5f);
	if (sl != 0 || !in_range) return;
	if (!(wi > 0.0f) || rc <= 0) { pout[idx] = p4; return; }
	const float inv_rec = 1.0f / (float)rc;
	const float3 avg = make_float3(sx * inv_rec, sy * inv_rec, sz * inv_rec);
	if (!fin3(avg)) { pout[idx] = p4; return; }
	const float3 o = gather_finish(pi, avg, __ldg(rest_len + idx), P->under_relax);
	pout[idx] = make_float4(o.x, o.y, o.z, p4.w);
}
// node of gather group g: order[g] when an order is given (nodes of similar reverse-list
// length side by side, so the groups of a warp run even trip counts)
__device__ __forceinline__ int ordered_node(const int* __restrict__ order, int g, int n)
{
	return (order && g < n) ? __ldg(order + g) : g;
}
// the 4-lane form is latency bound on its record loads: compiled for 6 resident blocks
// per SM (42 registers) it keeps more loads in flight (11.73 -> 11.46 ms per frame at 1M)
template <int S>
__global__ void __launch_bounds__(kBlock, S == 4 ? 6 : 1) k_volume_gather_group(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, float4* __restrict__ pout, const int* __restrict__ roff,
	const int* __restrict__ ridx, const float4* __restrict__ rec, const float* __restrict__ recz,
	const float* __restrict__ rest_len, const int* __restrict__ order)
{
	const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	gather_group_lane<S, true>((long long)ordered_node(order, (int)(g / S), n) * S + (g & (S - 1)), n, P, pin, pout,
		roff, ridx, rec, recz, rest_len);
}

// The distance, volume solve and gather kernels compiled for MINB resident blocks per SM
// (fewer registers, more warps in flight for these latency-bound gathers): the same
// per-item code, so the same results; the autotuner picks among the forms by timing.
template <int S, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_volume_gather_occ(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, float4* __restrict__ pout, const int* __restrict__ roff,
	const int* __restrict__ ridx, const float4* __restrict__ rec, const float* __restrict__ recz,
	const float* __restrict__ rest_len, const int* __restrict__ order)
{
	const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	gather_group_lane<S, true>((long long)ordered_node(order, (int)(g / S), n) * S + (g & (S - 1)), n, P, pin, pout,
		roff, ridx, rec, recz, rest_len);
}

// Kernel B, one thread per node (forward.cu:9187-9243)
__global__ void __launch_bounds__(kBlock) k_volume_gather_thread(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, float4* __restrict__ pout, const int* __restrict__ roff,
	const int* __restrict__ ridx, const float4* __restrict__ rec, const float* __restrict__ recz,
	const float* __restrict__ rest_len)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= n) return;
	const float4 p4 = ld4(pin, idx);
	const float3 pi = f3(p4);
	const float wi = p4.w * P->inv_mass_scale;
	if (wi <= 0.0f) { pout[idx] = p4; return; }
	float3 sum = make_float3(0.0f, 0.0f, 0.0f);
	int received = 0;
	for (int k = roff[idx]; k < roff[idx + 1]; ++k) {
		const int i = __ldg(ridx + k);
		if (i < 0 || i >= n) continue;
		float3 dp;
		if (!gather_one(rec, recz, i, pi, wi, dp)) continue;
		sum = add3(sum, dp);
		++received;
	}
	if (received <= 0) { pout[idx] = p4; return; }
	const float3 avg = mul3(sum, 1.0f / (float)received);
	if (!fin3(avg)) { pout[idx] = p4; return; }
	const float3 o = gather_finish(pi, avg, __ldg(rest_len + idx), P->under_relax);
	pout[idx] = make_float4(o.x, o.y, o.z, p4.w);
}

// volume Gauss-Seidel, one colour: thread per cluster, members moved in place with no
// averaging (forward.cu:9041-9183)
__global__ void __launch_bounds__(64) k_volume_gs(int begin, int count, const int* __restrict__ order, int n,
	const StepParams* __restrict__ P, float4* __restrict__ pos, const int* __restrict__ voff,
	const int* __restrict__ vidx, const float* __restrict__ det_rest, const int* __restrict__ mat_type,
	float* __restrict__ lam_vol, const float* __restrict__ rest_len, int read_lam)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= count) return;
	const int idx = order[begin + t];
	if (idx < 0 || idx >= n) return;
	if (mat_type[idx] != 0) return;
	const float4 p4 = pos[idx];
	const float3 pi = f3(p4);
	const int off = voff[idx], cnt = voff[idx + 1] - off;
	float3 c = pi;
	int used = 0;
	for (int k = 0; k < cnt; ++k) {
		const int j = vidx[off + k];
		if (j < 0 || j >= n) continue;
		c = add3(c, f3(pos[j]));
		++used;
	}
	if (used < 3) return;
	const float inv_n = 1.0f / (float)(used + 1);
	c = mul3(c, inv_n);
	M3 S;
	m3_zero(S);
	{
		const float3 d = sub3(pi, c);
		m3_add_outer(S, d, d);
	}
	for (int k = 0; k < cnt; ++k) {
		const int j = vidx[off + k];
		if (j < 0 || j >= n) continue;
		const float3 d = sub3(f3(pos[j]), c);
		m3_add_outer(S, d, d);
	}
#pragma unroll
	for (int cc = 0; cc < 3; ++cc)
#pragma unroll
		for (int r = 0; r < 3; ++r) S.m[cc][r] *= inv_n;
	float J, C;
	M3 Sinv;
	if (!cluster_j_sinv(S, det_rest[idx], J, C, Sinv)) return;
	const float gs = J * inv_n;
	const float ims = P->inv_mass_scale;
	float denom = 0.0f;
	{
		const float3 g = mul3(m3_mulv(Sinv, sub3(pi, c)), gs);
		denom += (p4.w * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
	}
	for (int k = 0; k < cnt; ++k) {
		const int j = vidx[off + k];
		if (j < 0 || j >= n) continue;
		const float4 q = pos[j];
		const float3 g = mul3(m3_mulv(Sinv, sub3(f3(q), c)), gs);
		denom += (q.w * ims) * (g.x * g.x + g.y * g.y + g.z * g.z);
	}
	const float dt = P->dt;
	const float dt2 = fmaxf(dt * dt, 1e-8f);
	const float alpha_t = P->vol_compliance / dt2;
	const float den = denom + alpha_t;
	if (!(den > 1e-12f)) return;
	const float lam = read_lam ? lam_vol[idx] : 0.0f;
	const float dl = (-C - alpha_t * lam) / den;
	if (!isfinite(dl)) return;
	lam_vol[idx] = lam + dl;
	const float coef = dl * gs;
	for (int k = -1; k < cnt; ++k) {
		const int j = (k < 0) ? idx : vidx[off + k];
		if (j < 0 || j >= n) continue;
		const float4 xj4 = pos[j];
		const float wj = xj4.w * ims;
		if (wj <= 0.0f) continue;
		const float3 xj = f3(xj4);
		const float3 g = m3_mulv(Sinv, sub3(xj, c));
		float3 dp = make_float3(g.x * wj * coef, g.y * wj * coef, g.z * wj * coef);
		if (!fin3(dp)) continue;
		const float rl = rest_len[j];
		if (rl > 1e-12f) {
			const float max_step = 0.25f * rl;
			const float len = len3(dp);
			if (len > max_step && len > 1e-20f) dp = mul3(dp, max_step / len);
		}
		const float3 o = add3(xj, dp);
		pos[j] = make_float4(o.x, o.y, o.z, xj4.w);
	}
}

// rest covariance, determinant, volume, rest length, material class per cluster
// (precomputeVolumeGaussianKernel, forward.cu:7691-7844; mixture rest off)
__global__ void __launch_bounds__(kBlock) k_volume_rest(int n, const float4* __restrict__ rest,
	const int* __restrict__ voff, const int* __restrict__ vidx, const int* __restrict__ goff,
	const int* __restrict__ gnbr, float aniso, float* __restrict__ sigma_rest, float* __restrict__ det_rest,
	float* __restrict__ v_rest, float* __restrict__ rest_len, int* __restrict__ mat_type)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= n) return;
	float* sig = sigma_rest + (size_t)idx * 6;
	for (int k = 0; k < 6; ++k) sig[k] = 0.0f;
	det_rest[idx] = 0.0f;
	v_rest[idx] = 0.0f;
	mat_type[idx] = 3;
	const float3 p0 = f3(rest[idx]);
	{
		float dmin = FLT_MAX;
		for (int e = goff[idx]; e < goff[idx + 1]; ++e) {
			const int j = gnbr[e];
			if (j < 0 || j >= n || j == idx) continue;
			const float dl = len3(sub3(f3(rest[j]), p0));
			if (dl > 1e-12f) dmin = fminf(dmin, dl);
		}
		rest_len[idx] = (dmin < FLT_MAX) ? dmin : 0.0f;
	}
	const int off = voff[idx], cnt = voff[idx + 1] - off;
	if (cnt < 4) return;
	float3 c = p0;
	int used = 0;
	for (int k = 0; k < cnt; ++k) {
		const int j = vidx[off + k];
		if (j < 0 || j >= n) continue;
		c = add3(c, f3(rest[j]));
		++used;
	}
	if (used < 3) return;
	const float inv_n = 1.0f / (float)(used + 1);
	c = mul3(c, inv_n);
	M3 S;
	m3_zero(S);
	{
		const float3 d = sub3(p0, c);
		m3_add_outer(S, d, d);
	}
	for (int k = 0; k < cnt; ++k) {
		const int j = vidx[off + k];
		if (j < 0 || j >= n) continue;
		const float3 d = sub3(f3(rest[j]), c);
		m3_add_outer(S, d, d);
	}
	for (int cc = 0; cc < 3; ++cc)
		for (int r = 0; r < 3; ++r) S.m[cc][r] *= inv_n;
	float s_rest, det_hat;
	if (!sigma_scale_det(S, s_rest, det_hat)) { mat_type[idx] = 4; return; }
	float3 eig;
	M3 V;
	eig_sym3f(S, eig, V);
	const float lmax = fmaxf(eig.z, 1e-24f);
	const float a1 = eig.x / lmax, a2 = eig.y / lmax;
	if (a1 > aniso) mat_type[idx] = 0;
	else if (a2 > aniso) mat_type[idx] = 1;
	else mat_type[idx] = 2;
	sig[0] = S.m[0][0]; sig[1] = S.m[1][1]; sig[2] = S.m[2][2];
	sig[3] = S.m[1][0]; sig[4] = S.m[2][0]; sig[5] = S.m[2][1];
	const float d = s_rest * s_rest * s_rest * det_hat;
	det_rest[idx] = d;
	v_rest[idx] = (4.0f / 3.0f) * 3.14159265f * sqrtf(fmaxf(d, 0.0f));
}

// ---------------------------------------------------------------------------
// shape matching over {i} + 1-ring (forward.cu:6088-6383), FP64 polar rotation
// (shapeMatchRotationDouble, forward.cu:5991-6086) or the float32 path
// (forward.cu:6238-6319); XPBD pull toward the goal (forward.cu:4972-4988).
// ---------------------------------------------------------------------------
// One cyclic-Jacobi rotation zeroing m[p][q] (p < q compile-time constants, so m and v
// stay in registers; a run-time pivot index would put them in local memory).
template <int p, int q>
__device__ __forceinline__ void jacobi_rotate_d(double (&m)[3][3], double (&v)[3][3])
{
	constexpr int r = 3 - p - q;
	const double app = m[p][p], aqq = m[q][q], apq = m[p][q];
	// t = sgn(phi) / (|phi| + sqrt(1 + phi^2)) with phi = (aqq - app) / (2 apq'), apq' =
	// apq + 1e-300, written as 2 |apq'| sgn / (|d| + sqrt(d^2 + 4 apq'^2)), d = aqq - app:
	// one division and one square root instead of two each (c from a reciprocal square
	// root).  Where d and apq' are both so small that their squares would underflow, the
	// phi form.
	const double d = aqq - app, h = apq + 1e-300;
	double t;
	if (fabs(d) > 1e-140 || fabs(h) > 1e-140) {
		const double sgn = (d == 0.0 || (d > 0.0) == (h > 0.0)) ? 1.0 : -1.0;
		t = sgn * (2.0 * fabs(h)) / (fabs(d) + sqrt(d * d + 4.0 * h * h));
	}
	else {
		const double phi = 0.5 * d / h;
		t = (phi >= 0.0) ? 1.0 / (phi + sqrt(1.0 + phi * phi)) : 1.0 / (phi - sqrt(1.0 + phi * phi));
	}
	const double c = rsqrt(1.0 + t * t);
	const double s = t * c;
	m[p][p] = app - t * apq;
	m[q][q] = aqq + t * apq;
	m[p][q] = m[q][p] = 0.0;
	const double arp = m[r][p], arq = m[r][q];
	m[r][p] = m[p][r] = c * arp - s * arq;
	m[r][q] = m[q][r] = c * arq + s * arp;
#pragma unroll
	for (int rr = 0; rr < 3; ++rr) {
		const double vrp = v[rr][p], vrq = v[rr][q];
		v[rr][p] = c * vrp - s * vrq;
		v[rr][q] = s * vrp + c * vrq;
	}
}

__device__ __forceinline__ bool shape_rotation_double(const M3& A, M3& Rout)
{
	double a[3][3];
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) a[r][c] = (double)A.m[c][r];
	double m[3][3];
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) m[r][c] = a[0][r] * a[0][c] + a[1][r] * a[1][c] + a[2][r] * a[2][c];
	double v[3][3] = { { 1.0, 0.0, 0.0 }, { 0.0, 1.0, 0.0 }, { 0.0, 0.0, 1.0 } };
	for (int iter = 0; iter < 50; ++iter) {
		bool done = true;
		int piv = 0;   // 0: (0,1), 1: (0,2), 2: (1,2)
		double max_off = -1.0;
#pragma unroll
		for (int k = 0; k < 3; ++k) {
			const int pk = (k == 2) ? 1 : 0, qk = (k == 0) ? 1 : 2;
			const double off = fabs(m[pk][qk]);
			// off > 1e-12 sqrt(|a_pp a_qq|) + 1e-300, compared in squares (no square root)
			if (off > 1e-300 && off * off > 1e-24 * fabs(m[pk][pk] * m[qk][qk])) done = false;
			if (off > max_off) { max_off = off; piv = k; }
		}
		if (done) break;
		if (piv == 0) jacobi_rotate_d<0, 1>(m, v);
		else if (piv == 1) jacobi_rotate_d<0, 2>(m, v);
		else jacobi_rotate_d<1, 2>(m, v);
	}
	double ev[3] = { m[0][0], m[1][1], m[2][2] };
#pragma unroll
	for (int i = 0; i < 2; ++i)
#pragma unroll
		for (int j = i + 1; j < 3; ++j)
			if (ev[i] > ev[j]) {
				const double te = ev[i]; ev[i] = ev[j]; ev[j] = te;
#pragma unroll
				for (int rr = 0; rr < 3; ++rr) { const double tv = v[rr][i]; v[rr][i] = v[rr][j]; v[rr][j] = tv; }
			}
	double S[3], Si[3];
#pragma unroll
	for (int i = 0; i < 3; ++i) S[i] = sqrt(ev[i] > 0.0 ? ev[i] : 0.0);
	const double smax = (S[2] > 1e-300) ? S[2] : 1e-300;
#pragma unroll
	for (int i = 0; i < 3; ++i) Si[i] = (S[i] > 1e-12 * smax) ? 1.0 / S[i] : 0.0;
	double u[3][3];
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) u[r][c] = (a[r][0] * v[0][c] + a[r][1] * v[1][c] + a[r][2] * v[2][c]) * Si[c];
	if (S[0] < 0.08 * smax) {
		const double cx = u[1][1] * u[2][2] - u[2][1] * u[1][2];
		const double cy = u[2][1] * u[0][2] - u[0][1] * u[2][2];
		const double cz = u[0][1] * u[1][2] - u[1][1] * u[0][2];
		const double len = sqrt(cx * cx + cy * cy + cz * cz);
		if (!(len > 1e-7)) return false;
		u[0][0] = cx / len; u[1][0] = cy / len; u[2][0] = cz / len;
	}
	double R[3][3];
	for (int pass = 0; pass < 2; ++pass) {
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) R[r][c] = u[r][0] * v[c][0] + u[r][1] * v[c][1] + u[r][2] * v[c][2];
		const double det = R[0][0] * (R[1][1] * R[2][2] - R[1][2] * R[2][1])
			- R[0][1] * (R[1][0] * R[2][2] - R[1][2] * R[2][0])
			+ R[0][2] * (R[1][0] * R[2][1] - R[1][1] * R[2][0]);
		if (det >= 0.0 || pass == 1) break;
#pragma unroll
		for (int rr = 0; rr < 3; ++rr) u[rr][0] = -u[rr][0];
	}
	bool ok = true;
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) {
			ok = ok && isfinite(R[r][c]);
			Rout.m[c][r] = (float)R[r][c];
		}
	return ok;
}

// shape_rotation_double with the Jacobi started from the eigenvector frame of this
// Gaussian's previous call (warm, a unit quaternion; all zero = identity) and that
// frame stored back.  The polar factor R = U V^T is unique for a non-singular A, so the
// start changes only where the iteration stops, not what it converges to (the same
// 1e-12 relative off-diagonal test); successive calls of one Gaussian see nearly the
// same A, which leaves one or two rotations instead of a full cold run.
__device__ __forceinline__ bool shape_rotation_double_warm(const M3& A, M3& Rout, float4& warm)
{
	double a[3][3];
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) a[r][c] = (double)A.m[c][r];
	double m[3][3];
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) m[r][c] = a[0][r] * a[0][c] + a[1][r] * a[1][c] + a[2][r] * a[2][c];
	double v[3][3] = { { 1.0, 0.0, 0.0 }, { 0.0, 1.0, 0.0 }, { 0.0, 0.0, 1.0 } };
	{
		double qw = warm.x, qx = warm.y, qy = warm.z, qz = warm.w;
		const double qn = qw * qw + qx * qx + qy * qy + qz * qz;
		if (qn > 0.5) {
			const double inv = 1.0 / sqrt(qn);
			qw *= inv; qx *= inv; qy *= inv; qz *= inv;
			v[0][0] = 1.0 - 2.0 * (qy * qy + qz * qz); v[0][1] = 2.0 * (qx * qy - qw * qz);
			v[0][2] = 2.0 * (qx * qz + qw * qy);
			v[1][0] = 2.0 * (qx * qy + qw * qz); v[1][1] = 1.0 - 2.0 * (qx * qx + qz * qz);
			v[1][2] = 2.0 * (qy * qz - qw * qx);
			v[2][0] = 2.0 * (qx * qz - qw * qy); v[2][1] = 2.0 * (qy * qz + qw * qx);
			v[2][2] = 1.0 - 2.0 * (qx * qx + qy * qy);
			// m <- V^T m V
			double t[3][3];
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c) t[r][c] = m[r][0] * v[0][c] + m[r][1] * v[1][c] + m[r][2] * v[2][c];
#pragma unroll
			for (int r = 0; r < 3; ++r)
#pragma unroll
				for (int c = 0; c < 3; ++c) m[r][c] = v[0][r] * t[0][c] + v[1][r] * t[1][c] + v[2][r] * t[2][c];
		}
	}
	for (int iter = 0; iter < 50; ++iter) {
		bool done = true;
		int piv = 0;   // 0: (0,1), 1: (0,2), 2: (1,2)
		double max_off = -1.0;
#pragma unroll
		for (int k = 0; k < 3; ++k) {
			const int pk = (k == 2) ? 1 : 0, qk = (k == 0) ? 1 : 2;
			const double off = fabs(m[pk][qk]);
			// off > 1e-12 sqrt(|a_pp a_qq|) + 1e-300, compared in squares (no square root)
			if (off > 1e-300 && off * off > 1e-24 * fabs(m[pk][pk] * m[qk][qk])) done = false;
			if (off > max_off) { max_off = off; piv = k; }
		}
		if (done) break;
		if (piv == 0) jacobi_rotate_d<0, 1>(m, v);
		else if (piv == 1) jacobi_rotate_d<0, 2>(m, v);
		else jacobi_rotate_d<1, 2>(m, v);
	}
	{
		// the converged frame (a proper rotation: products of rotations), as a unit
		// quaternion for the next call (largest-component extraction).  Kept in FP32: it
		// only seeds the next call's Jacobi (re-normalised in FP64 there), whose stop test
		// decides the result
		float f[3][3];
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) f[r][c] = (float)v[r][c];
		const float tr = f[0][0] + f[1][1] + f[2][2];
		float qw, qx, qy, qz;
		if (tr > 0.0f) {
			const float s2 = 2.0f * sqrtf(1.0f + tr), r2 = 1.0f / s2;
			qw = 0.25f * s2; qx = (f[2][1] - f[1][2]) * r2; qy = (f[0][2] - f[2][0]) * r2; qz = (f[1][0] - f[0][1]) * r2;
		} else if (f[0][0] > f[1][1] && f[0][0] > f[2][2]) {
			const float s2 = 2.0f * sqrtf(fmaxf(1.0f + f[0][0] - f[1][1] - f[2][2], 1e-30f)), r2 = 1.0f / s2;
			qw = (f[2][1] - f[1][2]) * r2; qx = 0.25f * s2; qy = (f[0][1] + f[1][0]) * r2; qz = (f[0][2] + f[2][0]) * r2;
		} else if (f[1][1] > f[2][2]) {
			const float s2 = 2.0f * sqrtf(fmaxf(1.0f + f[1][1] - f[0][0] - f[2][2], 1e-30f)), r2 = 1.0f / s2;
			qw = (f[0][2] - f[2][0]) * r2; qx = (f[0][1] + f[1][0]) * r2; qy = 0.25f * s2; qz = (f[1][2] + f[2][1]) * r2;
		} else {
			const float s2 = 2.0f * sqrtf(fmaxf(1.0f + f[2][2] - f[0][0] - f[1][1], 1e-30f)), r2 = 1.0f / s2;
			qw = (f[1][0] - f[0][1]) * r2; qx = (f[0][2] + f[2][0]) * r2; qy = (f[1][2] + f[2][1]) * r2; qz = 0.25f * s2;
		}
		warm = isfinite(qw + qx + qy + qz) ? make_float4(qw, qx, qy, qz) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	}
	double ev[3] = { m[0][0], m[1][1], m[2][2] };
#pragma unroll
	for (int i = 0; i < 2; ++i)
#pragma unroll
		for (int j = i + 1; j < 3; ++j)
			if (ev[i] > ev[j]) {
				const double te = ev[i]; ev[i] = ev[j]; ev[j] = te;
#pragma unroll
				for (int rr = 0; rr < 3; ++rr) { const double tv = v[rr][i]; v[rr][i] = v[rr][j]; v[rr][j] = tv; }
			}
	// singular values and their inverses from one reciprocal square root each (in place
	// of a square root and a division: equal to FP64 rounding)
	double S[3], Si[3];
#pragma unroll
	for (int i = 0; i < 3; ++i) {
		Si[i] = ev[i] > 0.0 ? rsqrt(ev[i]) : 0.0;
		S[i] = ev[i] > 0.0 ? ev[i] * Si[i] : 0.0;
	}
	const double smax = (S[2] > 1e-300) ? S[2] : 1e-300;
#pragma unroll
	for (int i = 0; i < 3; ++i) Si[i] = (S[i] > 1e-12 * smax) ? Si[i] : 0.0;
	double u[3][3];
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) u[r][c] = (a[r][0] * v[0][c] + a[r][1] * v[1][c] + a[r][2] * v[2][c]) * Si[c];
	if (S[0] < 0.08 * smax) {
		const double cx = u[1][1] * u[2][2] - u[2][1] * u[1][2];
		const double cy = u[2][1] * u[0][2] - u[0][1] * u[2][2];
		const double cz = u[0][1] * u[1][2] - u[1][1] * u[0][2];
		const double len = sqrt(cx * cx + cy * cy + cz * cz);
		if (!(len > 1e-7)) return false;
		u[0][0] = cx / len; u[1][0] = cy / len; u[2][0] = cz / len;
	}
	double R[3][3];
	for (int pass = 0; pass < 2; ++pass) {
#pragma unroll
		for (int r = 0; r < 3; ++r)
#pragma unroll
			for (int c = 0; c < 3; ++c) R[r][c] = u[r][0] * v[c][0] + u[r][1] * v[c][1] + u[r][2] * v[c][2];
		const double det = R[0][0] * (R[1][1] * R[2][2] - R[1][2] * R[2][1])
			- R[0][1] * (R[1][0] * R[2][2] - R[1][2] * R[2][0])
			+ R[0][2] * (R[1][0] * R[2][1] - R[1][1] * R[2][0]);
		if (det >= 0.0 || pass == 1) break;
#pragma unroll
		for (int rr = 0; rr < 3; ++rr) u[rr][0] = -u[rr][0];
	}
	bool ok = true;
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) {
			ok = ok && isfinite(R[r][c]);
			Rout.m[c][r] = (float)R[r][c];
		}
	return ok;
}

__device__ __noinline__ bool shape_rotation_float(const M3& A, M3& Rout)
{
	const M3 AtA = m3_mul(m3_t(A), A);
	float3 S2;
	M3 V;
	eig_sym3f(AtA, S2, V);
	const float3 Sv = make_float3(sqrtf(fmaxf(0.0f, S2.x)), sqrtf(fmaxf(0.0f, S2.y)), sqrtf(fmaxf(0.0f, S2.z)));
	if (!fin3(Sv)) return false;
	M3 Si;
	m3_zero(Si);
	Si.m[0][0] = (Sv.x > 1e-7f) ? 1.0f / Sv.x : 0.0f;
	Si.m[1][1] = (Sv.y > 1e-7f) ? 1.0f / Sv.y : 0.0f;
	Si.m[2][2] = (Sv.z > 1e-7f) ? 1.0f / Sv.z : 0.0f;
	M3 U = m3_mul(m3_mul(A, V), Si);
	if (!m3_finite(U)) return false;
	if (Sv.x < 0.08f * fmaxf(Sv.z, 1e-7f)) {
		const float3 u1 = make_float3(U.m[1][0], U.m[1][1], U.m[1][2]);
		const float3 u2 = make_float3(U.m[2][0], U.m[2][1], U.m[2][2]);
		const float3 cr = make_float3(u1.y * u2.z - u2.y * u1.z, u1.z * u2.x - u2.z * u1.x, u1.x * u2.y - u2.x * u1.y);
		const float l = sqrtf(dot3(cr, cr));
		if (!(l > 1e-7f)) return false;
		U.m[0][0] = cr.x / l; U.m[0][1] = cr.y / l; U.m[0][2] = cr.z / l;
	}
	const M3 Vt = m3_t(V);
	M3 R = m3_mul(U, Vt);
	if (!m3_finite(R)) return false;
	if (m3_det(R) < 0.0f) {
		U.m[0][0] *= -1.0f; U.m[0][1] *= -1.0f; U.m[0][2] *= -1.0f;
		R = m3_mul(U, Vt);
		if (!m3_finite(R)) return false;
	}
	Rout = R;
	return true;
}

// Rest-state part of shape matching, fixed for the life of the graph: the rest centroid
// of {i} + 1-ring, 1 / member count, and the skips that depend only on the rest pose and
// the topology (fewer than 4 neighbours, boundary bias > 0.4; forward.cu:6116-6176).
// out[i] = (rest centroid, 1 / count), or w = -1 when node i is never shape-matched.
__global__ void __launch_bounds__(kBlock) k_shape_rest(int n, const float4* __restrict__ rest,
	const int* __restrict__ off, const int* __restrict__ nbr, float4* __restrict__ out)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= n) return;
	const float4 skip = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
	const int e0 = off[idx], e1 = off[idx + 1];
	const int cnt = e1 - e0;
	if (cnt < 4) { out[idx] = skip; return; }
	float3 com_rest = f3(ld4(rest, idx));
	float cluster_count = 1.0f;
	for (int e = e0; e < e1; ++e) {
		const int j = __ldg(nbr + e);
		if (j < 0 || j >= n) continue;
		com_rest = add3(com_rest, f3(ld4(rest, j)));
		cluster_count += 1.0f;
	}
	if (cluster_count < 2.0f) { out[idx] = skip; return; }
	const float inv_c = 1.0f / cluster_count;
	com_rest = mul3(com_rest, inv_c);
	float3 dir_sum = make_float3(0.0f, 0.0f, 0.0f);
	for (int e = e0; e < e1; ++e) {
		const int j = __ldg(nbr + e);
		if (j < 0 || j >= n) continue;
		const float3 q = sub3(f3(ld4(rest, j)), com_rest);
		const float len = len3(q);
		if (len > 1e-7f) dir_sum = add3(dir_sum, mul3(q, 1.0f / len));
	}
	const float bias = len3(dir_sum) / fmaxf((float)cnt, 1.0f);
	if (bias > 0.4f) { out[idx] = skip; return; }
	out[idx] = make_float4(com_rest.x, com_rest.y, com_rest.z, inv_c);
}

// Per-iteration shape matching: current centroid, A = sum (p - c)(q - c_rest)^T over
// {i} + 1-ring, normalised, rotation by polar decomposition (FP64 Jacobi when ROBUST,
// else float), goal projection.  The rest-only terms come from k_shape_rest.  Three
// blocks per SM (80 registers, a few spilled) hide more of the FP64 Jacobi chain's
// latency than two (measured 1.3 -> 1.05 ms per substep at 1M).
template <bool ROBUST, bool NC>
__device__ __forceinline__ void shape_row(int idx, int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, float4* __restrict__ pout, const float4* __restrict__ rest,
	const int* __restrict__ off, const int* __restrict__ nbr, const float4* __restrict__ shape_rest,
	float4* __restrict__ shape_q)
{
	if (idx >= n) return;
	const float4 p4 = ldv<NC>(pin, idx);
	const float3 pi = f3(p4);
	const float wi = p4.w * P->inv_mass_scale;
	if (wi <= 0.0f) { pout[idx] = p4; return; }
	const float4 sr = ld4(shape_rest, idx);
	if (!(sr.w > 0.0f)) { pout[idx] = p4; return; }
	const int e0 = off[idx], e1 = off[idx + 1];
	const float3 ri = f3(ld4(rest, idx));
	const float3 com_rest = f3(sr);
	// one pass over the 1-ring, two neighbours per trip (loads in flight together):
	// the current centroid's sum in row order (as the two-pass form computes it) and,
	// relative to the Gaussian itself (dq = q - p_i, dr = r - r_i), the sums of dq, dr
	// and dq dr^T.  With cq = com - p_i and cr = com_rest - r_i,
	//   A = sum_k (q_k - com)(r_k - com_rest)^T = sum dq dr^T - cq (sum dr)^T - (sum dq) cr^T
	//       + (m+1) cq cr^T
	// over the Gaussian and its m neighbours (the Gaussian's own dq = dr = 0); the
	// neighbours lie within a spacing or two, so the shifted moments lose little to
	// cancellation (equal to the two-pass sums to FP32 rounding).
	float3 sq = pi, sdq = make_float3(0.0f, 0.0f, 0.0f), sdr = sdq;
	float count = 1.0f;
	M3 A;
	m3_zero(A);
	auto add = [&](float4 q, float4 r) {
		sq = add3(sq, f3(q));
		const float3 dq = sub3(f3(q), pi), dr = sub3(f3(r), ri);
		sdq = add3(sdq, dq);
		sdr = add3(sdr, dr);
		m3_add_outer(A, dq, dr);
		count += 1.0f;
	};
	int e = e0;
	for (; e + 1 < e1; e += 2) {
		const int j0 = __ldg(nbr + e), j1 = __ldg(nbr + e + 1);
		const bool ok0 = j0 >= 0 && j0 < n, ok1 = j1 >= 0 && j1 < n;
		float4 q0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), q1 = q0, r0 = q0, r1 = q0;
		if (ok0) { q0 = ldv<NC>(pin, j0); r0 = ld4(rest, j0); }
		if (ok1) { q1 = ldv<NC>(pin, j1); r1 = ld4(rest, j1); }
		if (ok0) add(q0, r0);
		if (ok1) add(q1, r1);
	}
	if (e < e1) {
		const int j = __ldg(nbr + e);
		if (j >= 0 && j < n) add(ldv<NC>(pin, j), ld4(rest, j));
	}
	const float3 com_curr = mul3(sq, sr.w);
	const float3 cq = sub3(com_curr, pi), cr = sub3(com_rest, ri);
	m3_add_outer(A, cq, mul3(sdr, -1.0f));
	m3_add_outer(A, mul3(sdq, -1.0f), cr);
	m3_add_outer(A, mul3(cq, count), cr);
	float a_norm_sq = 0.0f;
#pragma unroll
	for (int c = 0; c < 3; ++c)
#pragma unroll
		for (int r = 0; r < 3; ++r) a_norm_sq += A.m[c][r] * A.m[c][r];
	const float a_norm = sqrtf(a_norm_sq);
	if (!isfinite(a_norm) || a_norm < 1e-8f) { pout[idx] = p4; return; }
#pragma unroll
	for (int c = 0; c < 3; ++c)
#pragma unroll
		for (int r = 0; r < 3; ++r) A.m[c][r] /= a_norm;
	M3 R;
	bool ok;
	if (ROBUST) {
		float4 q = shape_q[idx];
		ok = shape_rotation_double_warm(A, R, q);
		shape_q[idx] = q;
	}
	else {
		ok = shape_rotation_float(A, R);
	}
	if (!ok) { pout[idx] = p4; return; }
	const float3 goal = add3(com_curr, m3_mulv(R, sub3(ri, com_rest)));
	const float3 gd = sub3(goal, pi);
	const float gd2 = dot3(gd, gd);
	if (!isfinite(gd2) || gd2 < 1e-18f) { pout[idx] = p4; return; }
	const float dt = P->dt;
	const float dt2 = fmaxf(dt * dt, 1e-8f);
	const float alpha_tilde = P->shape_compliance / dt2;
	const float denom = wi + alpha_tilde;
	if (denom < 1e-8f) { pout[idx] = p4; return; }
	const float scale = P->shape_blend * (wi / denom);
	const float3 o = add3(pi, mul3(sub3(goal, pi), scale));
	pout[idx] = make_float4(o.x, o.y, o.z, p4.w);
}
// four resident blocks per SM (64 registers, some spills): more warps hide the FP64
// chain's latency better than fewer spills (measured against three and five)
template <bool ROBUST>
__global__ void __launch_bounds__(kBlock, 4) k_shape_match(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pin, float4* __restrict__ pout, const float4* __restrict__ rest,
	const int* __restrict__ off, const int* __restrict__ nbr, const float4* __restrict__ shape_rest,
	float4* __restrict__ shape_q)
{
	shape_row<ROBUST, true>(blockIdx.x * blockDim.x + threadIdx.x, n, P, pin, pout, rest, off, nbr, shape_rest, shape_q);
}

// ---------------------------------------------------------------------------
// per-Gaussian projections at the end of an iteration: self-collision apply
// (forward.cu:7311-7322), kinematic colliders (forward.cu:7425-7518) and the ground
// plane (forward.cu:7405-7421), fused in that order.  With ellipsoid contact shapes
// (cshape / crmax non-null) a collider's reach grows by the Gaussian's longest
// semi-axis and its distance shrinks by the support along the contact normal; with
// ground contact shapes (crg non-null) the plane is offset by the support radius.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void project_row(int idx, int n, const StepParams* __restrict__ P, float4* __restrict__ pos,
	const float4* __restrict__ pos_start, const int* __restrict__ sc_count, const float4* __restrict__ sc_dp,
	DevCounters* __restrict__ ctr, int count_hits, const int* __restrict__ obj_id,
	const KinCollider* __restrict__ ext_kin, const int2* __restrict__ ext_range, const float4* __restrict__ sc_dp_cross,
	float4* __restrict__ sc_accum, const float4* __restrict__ cshape, const float* __restrict__ crmax,
	const float* __restrict__ crg)
{
	if (idx >= n) return;
	float4 p4 = pos[idx];
	bool moved = false;
	// press plates (squashPressProjectKernel, forward.cu:9411-9424): a centre outside
	// [lo, hi] on the load axis goes onto the plate; the other axes are free (no friction)
	if (P->press_on && p4.w > 0.0f) {
		const int ax = P->press_axis;
		const float v = ax == 0 ? p4.x : (ax == 1 ? p4.y : p4.z);
		if (v < P->press_lo || v > P->press_hi) {
			const float t = v < P->press_lo ? P->press_lo : P->press_hi;
			if (ax == 0) p4.x = t;
			else if (ax == 1) p4.y = t;
			else p4.z = t;
			moved = true;
		}
	}
	if (sc_count && sc_count[idx] > 0) {
		const float4 d = sc_dp[idx];
		p4.x = p4.x + d.x; p4.y = p4.y + d.y; p4.z = p4.z + d.z;
		moved = true;
		if (sc_accum) {   // the frame's cross-object part, for the contact push (forward.cu:7311-7322)
			const float4 c = sc_dp_cross[idx];
			float4 a = sc_accum[idx];
			a.x = a.x + c.x; a.y = a.y + c.y; a.z = a.z + c.z;
			sc_accum[idx] = a;
		}
	}
	if (p4.w > 0.0f) {
		float3 p = f3(p4);
		const float margin = P->kin_margin, mu = P->kin_friction;
		const float rmax = crmax ? crmax[idx] : 0.0f;
		const float reach = margin + rmax;   // a centre farther than this keeps its ellipsoid clear too
		const int my_obj = ((P->kin_filtered || ext_kin) && obj_id) ? obj_id[idx] : -1;
		// colliders: the reference's list (with optional per-collider object filter), or the
		// batched list sorted by object, of which only this object's range is visited
		const KinCollider* cols = P->kin;
		int c0 = 0, c1 = P->kin_count;
		if (ext_kin) {
			cols = ext_kin;
			c0 = c1 = 0;
			if (my_obj >= 0 && my_obj < P->kin_ext_ranges) {
				const int2 r = ext_range[my_obj];
				c0 = r.x;
				c1 = r.y;
			}
		}
		for (int c = c0; c < c1; ++c) {
			const KinCollider& C = cols[c];
			if (C.obj >= 0 && C.obj != my_obj) continue;
			const float dx = p.x - C.t[0], dy = p.y - C.t[1], dz = p.z - C.t[2];
			const float lx = C.R[0] * dx + C.R[3] * dy + C.R[6] * dz;
			const float ly = C.R[1] * dx + C.R[4] * dy + C.R[7] * dz;
			const float lz = C.R[2] * dx + C.R[5] * dy + C.R[8] * dz;
			// (lx, ly, lz): the point in the collider frame; (nx, ny, nz): the outward normal
			// there; dist: the signed distance to the surface
			float nx = 0.0f, ny = 0.0f, nz = 1.0f, dist;
			if (C.type == 1) {   // box: excess over the half extents, its positive part outside
				const float ex = fabsf(lx) - C.h[0], ey = fabsf(ly) - C.h[1], ez = fabsf(lz) - C.h[2];
				if (ex > 0.0f || ey > 0.0f || ez > 0.0f) {
					const float bx = fmaxf(ex, 0.0f), by = fmaxf(ey, 0.0f), bz = fmaxf(ez, 0.0f);
					dist = sqrtf(bx * bx + by * by + bz * bz);
					if (dist >= reach) continue;
					const float inv = 1.0f / fmaxf(dist, 1e-20f);
					nx = copysignf(bx * inv, lx); ny = copysignf(by * inv, ly); nz = copysignf(bz * inv, lz);
				}
				else {
					if (ex >= ey && ex >= ez) { dist = ex; nx = (lx >= 0.0f) ? 1.0f : -1.0f; nz = 0.0f; }
					else if (ey >= ez) { dist = ey; ny = (ly >= 0.0f) ? 1.0f : -1.0f; nz = 0.0f; }
					else { dist = ez; nz = (lz >= 0.0f) ? 1.0f : -1.0f; }
				}
			}
			else {   // sphere (type 0) or capsule (type 2: segment along local z, half length h[1])
				float az = lz;
				if (C.type == 2) az = lz - fminf(fmaxf(lz, -C.h[1]), C.h[1]);
				const float rad = sqrtf(lx * lx + ly * ly + az * az);
				dist = rad - C.h[0];
				if (dist >= reach) continue;
				if (rad > 1e-20f) { nx = lx / rad; ny = ly / rad; nz = az / rad; }
			}
			const float wx = C.R[0] * nx + C.R[1] * ny + C.R[2] * nz;
			const float wy = C.R[3] * nx + C.R[4] * ny + C.R[5] * nz;
			const float wz = C.R[6] * nx + C.R[7] * ny + C.R[8] * nz;
			if (crmax && rmax > 0.0f) {   // the ellipsoid reaches that much closer along the normal
				dist -= contact_support(cshape[2 * idx], cshape[2 * idx + 1], wx, wy, wz);
				if (dist >= margin) continue;
			}
			const float corr = margin - dist;
			const float3 p_in = p;
			// explicit roundings: the batched-list and reference-list paths of this loop
			// must round identically, whatever the compiler fuses in each
			float3 dp = make_float3(__fmul_rn(wx, corr), __fmul_rn(wy, corr), __fmul_rn(wz, corr));
			p.x = __fadd_rn(p.x, dp.x); p.y = __fadd_rn(p.y, dp.y); p.z = __fadd_rn(p.z, dp.z);
			if (mu > 0.0f) {
				const float ox = C.Rp[0] * lx + C.Rp[1] * ly + C.Rp[2] * lz + C.tp[0];
				const float oy = C.Rp[3] * lx + C.Rp[4] * ly + C.Rp[5] * lz + C.tp[1];
				const float oz = C.Rp[6] * lx + C.Rp[7] * ly + C.Rp[8] * lz + C.tp[2];
				const float4 x0 = pos_start[idx];
				const float rx = (p.x - x0.x) - (p_in.x - ox), ry = (p.y - x0.y) - (p_in.y - oy),
					rz = (p.z - x0.z) - (p_in.z - oz);
				const float rn = rx * wx + ry * wy + rz * wz;
				const float tx = rx - rn * wx, ty = ry - rn * wy, tz = rz - rn * wz;
				const float lt = sqrtf(tx * tx + ty * ty + tz * tz);
				if (lt > 1e-20f) {
					const float k = fminf(1.0f, mu * corr / lt);
					const float fx = __fmul_rn(k, tx), fy = __fmul_rn(k, ty), fz = __fmul_rn(k, tz);
					p.x = __fsub_rn(p.x, fx); p.y = __fsub_rn(p.y, fy); p.z = __fsub_rn(p.z, fz);
					dp.x = __fsub_rn(dp.x, fx); dp.y = __fsub_rn(dp.y, fy); dp.z = __fsub_rn(dp.z, fz);
				}
			}
			moved = true;
			if (!ext_kin) {   // per-collider statistics cover the reference's list only
				float* acc = &ctr->kin_push[kColliderAcc * c];
				const float w = sqrtf(dp.x * dp.x + dp.y * dp.y + dp.z * dp.z);
				atomicAdd(&acc[0], dp.x);
				atomicAdd(&acc[1], dp.y);
				atomicAdd(&acc[2], dp.z);
				atomicAdd(&acc[3], w * p.x);
				atomicAdd(&acc[4], w * p.y);
				atomicAdd(&acc[5], w * p.z);
				atomicAdd(&acc[6], w);
				if (count_hits) atomicAdd(&ctr->kin_hits[c], 1);
			}
		}
		if (P->ground_on) {
			const float c = P->gn[0] * p.x + P->gn[1] * p.y + P->gn[2] * p.z - P->ground_plane - (crg ? crg[idx] : 0.0f);
			if (c < 0.0f) {
				p = make_float3(p.x - c * P->gn[0], p.y - c * P->gn[1], p.z - c * P->gn[2]);
				moved = true;
			}
		}
		p4.x = p.x; p4.y = p.y; p4.z = p.z;
	}
	if (moved) pos[idx] = p4;
}
__global__ void __launch_bounds__(kBlock) k_project(int n, const StepParams* __restrict__ P, float4* __restrict__ pos,
	const float4* __restrict__ pos_start, const int* __restrict__ sc_count, const float4* __restrict__ sc_dp,
	DevCounters* __restrict__ ctr, int count_hits, const int* __restrict__ obj_id,
	const KinCollider* __restrict__ ext_kin, const int2* __restrict__ ext_range, const float4* __restrict__ sc_dp_cross,
	float4* __restrict__ sc_accum, const float4* __restrict__ cshape, const float* __restrict__ crmax,
	const float* __restrict__ crg)
{
	project_row(blockIdx.x * blockDim.x + threadIdx.x, n, P, pos, pos_start, sc_count, sc_dp, ctr, count_hits, obj_id,
		ext_kin, ext_range, sc_dp_cross, sc_accum, cshape, crmax, crg);
}

// ---------------------------------------------------------------------------
// velocity commit (forward.cu:6623-6672) and its ground variant (forward.cu:7528-7599);
// also refreshes the caller-layout float3 position mirror.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void velocity_row(int idx, int n, const StepParams* __restrict__ P,
	float4* __restrict__ pos_curr, const float4* __restrict__ pfinal, float4* __restrict__ vel,
	float* __restrict__ pos_out3, const int* __restrict__ perm, const float* __restrict__ crg)
{
	if (idx >= n) return;
	const float4 x4 = pos_curr[idx];
	const float4 p4 = pfinal[idx];
	const float3 x = f3(x4), p = f3(p4);
	const float w = p4.w;
	const float dt = P->dt;
	float3 v = make_float3(0.0f, 0.0f, 0.0f);
	if (!P->ground_on) {
		if (w > 0.0f) {
			const float3 dx = sub3(p, x);
			const float dx2 = dot3(dx, dx);
			if (isfinite(dx2) && !(dx2 < 1e-18f)) {
				v = mul3(dx, 1.0f / fmaxf(dt, 1e-8f));
				const float damping = fminf(fmaxf(P->vel_damping, 0.0f), 1.0f);
				v = mul3(v, 1.0f - damping);
				if (!fin3(v) || dot3(v, v) < 1e-16f) v = make_float3(0.0f, 0.0f, 0.0f);
			}
		}
	}
	else if (w > 0.0f) {
		const float3 v_pre = f3(vel[idx]);
		const float3 dx = sub3(p, x);
		const float dx2 = dot3(dx, dx);
		if (isfinite(dx2)) {
			v = (dx2 < 1e-18f) ? make_float3(0.0f, 0.0f, 0.0f) : mul3(dx, 1.0f / fmaxf(dt, 1e-8f));
			const float3 nn = make_float3(P->gn[0], P->gn[1], P->gn[2]);
			const float gap = nn.x * p.x + nn.y * p.y + nn.z * p.z - P->ground_plane - (crg ? crg[idx] : 0.0f);
			if (gap <= P->ground_slop) {
				const float vn = nn.x * v.x + nn.y * v.y + nn.z * v.z;
				const float vn_pre = nn.x * v_pre.x + nn.y * v_pre.y + nn.z * v_pre.z;
				float vn_new = vn, jn = 0.0f;
				if (vn_pre < 0.0f) {
					const float e = (-vn_pre <= P->resting_speed) ? 0.0f : P->ground_restitution;
					vn_new = fmaxf(vn, -e * vn_pre);
					jn = -(1.0f + e) * vn_pre;
				}
				float3 vt = make_float3(v.x - vn * nn.x, v.y - vn * nn.y, v.z - vn * nn.z);
				const float vt_len = len3(vt);
				const float dvt = P->ground_friction * jn;
				if (vt_len <= dvt || vt_len < 1e-12f) vt = make_float3(0.0f, 0.0f, 0.0f);
				else vt = mul3(vt, (vt_len - dvt) / vt_len);
				v = make_float3(vt.x + vn_new * nn.x, vt.y + vn_new * nn.y, vt.z + vn_new * nn.z);
			}
			const float damping = fminf(fmaxf(P->vel_damping, 0.0f), 1.0f);
			v = mul3(v, 1.0f - damping);
			if (!fin3(v) || dot3(v, v) < 1e-16f) v = make_float3(0.0f, 0.0f, 0.0f);
		}
	}
	vel[idx] = make_float4(v.x, v.y, v.z, 0.0f);
	pos_curr[idx] = p4;
	if (pos_out3) {
		const size_t o = 3 * (size_t)(perm ? perm[idx] : idx);
		pos_out3[o + 0] = p.x;
		pos_out3[o + 1] = p.y;
		pos_out3[o + 2] = p.z;
	}
}
__global__ void __launch_bounds__(kBlock) k_velocity(int n, const StepParams* __restrict__ P,
	float4* __restrict__ pos_curr, const float4* __restrict__ pfinal, float4* __restrict__ vel,
	float* __restrict__ pos_out3, const int* __restrict__ perm, const float* __restrict__ crg)
{
	velocity_row(blockIdx.x * blockDim.x + threadIdx.x, n, P, pos_curr, pfinal, vel, pos_out3, perm, crg);
}

// ---------------------------------------------------------------------------
// self-collision (forward.cu:6984-7322, 11796-11849), spatial hash of the step's start
// positions, stable counting sort (same order as a stable radix sort of (key, index)),
// per-particle candidate lists, and the two-phase per-iteration solve.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned int sc_hash(int cx, int cy, int cz, unsigned int mask)
{
	return (((unsigned int)cx * 73856093u) ^ ((unsigned int)cy * 19349663u) ^ ((unsigned int)cz * 83492791u)) & mask;
}
__device__ __forceinline__ int sc_cell(float v, float inv_cell)
{
	return (int)floorf(fminf(fmaxf(v * inv_cell, -1.0e9f), 1.0e9f));
}

// The hashes of the 27 cells around (cx, cy, cz) in the reference's order kc = 9 (dz + 1)
// + 3 (dy + 1) + (dx + 1): sc_hash(cx + dx, cy + dy, cz + dz) = ((cx P1 + dx P1) ^ ...)
// in 32-bit wrap-around arithmetic, so the per-axis products are formed once and a cell
// costs three multiply-adds, two XORs and the mask (kc decoded without division).
struct Hash27 {
	unsigned int bx, by, bz, mask;
	__device__ __forceinline__ Hash27(int cx, int cy, int cz, unsigned int m)
		: bx((unsigned int)cx * 73856093u), by((unsigned int)cy * 19349663u), bz((unsigned int)cz * 83492791u),
		  mask(m)
	{
	}
	__device__ __forceinline__ unsigned int operator()(int kc) const
	{
		const int q = (kc * 11) >> 5;   // kc / 3 for kc < 27
		const int iz = (kc * 57) >> 9;  // kc / 9
		const int ix = kc - 3 * q, iy = q - 3 * iz;
		return ((bx + (unsigned int)(ix - 1) * 73856093u) ^ (by + (unsigned int)(iy - 1) * 19349663u) ^
			(bz + (unsigned int)(iz - 1) * 83492791u)) & mask;
	}
};

// bit kc set for the cells whose hash repeats no earlier cell's (the reference visits a
// bucket once, forward.cu:7116-7123); a 64-bit filter on the low hash bits settles
// almost every test without comparing, the rest compare with the earlier hashes
__device__ __forceinline__ unsigned int hash27_unique(const Hash27& H)
{
	unsigned int use = 0u;
	unsigned long long seen = 0ull;
#pragma unroll
	for (int kc = 0; kc < 27; ++kc) {
		const unsigned int h = H(kc);
		const unsigned long long bit = 1ull << (h & 63u);
		if (seen & bit) {
			bool dup = false;
			for (int m = 0; m < kc && !dup; ++m) dup = H(m) == h;
			if (dup) continue;
		}
		seen |= bit;
		use |= 1u << kc;
	}
	return use;
}

// order-preserving unsigned image of a (non-NaN) float, for atomicMax
__device__ __forceinline__ unsigned int f_order(float v)
{
	const unsigned int b = __float_as_uint(v);
	return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float f_unorder(unsigned int u)
{
	return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// max predict displacement^2 (selfColDispKernel + DeviceReduce::Max); with `bounds`,
// also the box of the predicted positions of the particles in the grid (active, start
// and predicted position finite) for the near-pair grid: order-preserving images, the
// minimum complemented, so that both ends are atomicMax on zero-initialised counters.
// Grid-stride over the particles, one set of atomics per block.
__global__ void __launch_bounds__(kBlock) k_sc_disp(int n, const float4* __restrict__ x, const float4* __restrict__ p,
	DevCounters* __restrict__ ctr, const unsigned char* __restrict__ active, int bounds)
{
	unsigned int m[7] = { 0u, 0u, 0u, 0u, 0u, 0u, 0u };   // disp^2 bits, lo x y z, hi x y z
	for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
		if (active && !active[i]) continue;
		const float4 a = x[i], b = p[i];
		const float dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
		const float v = dx * dx + dy * dy + dz * dz;
		m[0] = max(m[0], __float_as_uint(isfinite(v) ? v : 0.0f));
		if (bounds && isfinite(a.x) && isfinite(a.y) && isfinite(a.z) && isfinite(b.x) && isfinite(b.y) &&
			isfinite(b.z)) {
			const float c[3] = { b.x, b.y, b.z };
#pragma unroll
			for (int k = 0; k < 3; ++k) { m[1 + k] = max(m[1 + k], ~f_order(c[k])); m[4 + k] = max(m[4 + k], f_order(c[k])); }
		}
	}
	__shared__ unsigned int sm[7][kBlock / 32];
#pragma unroll
	for (int k = 0; k < 7; ++k) {
		for (int o = 16; o > 0; o >>= 1) m[k] = max(m[k], __shfl_xor_sync(0xffffffffu, m[k], o));
		if ((threadIdx.x & 31) == 0) sm[k][threadIdx.x >> 5] = m[k];
	}
	__syncthreads();
	if (threadIdx.x < 32) {
#pragma unroll
		for (int k = 0; k < 7; ++k) {
			unsigned int v = (threadIdx.x < blockDim.x / 32) ? sm[k][threadIdx.x] : 0u;
			for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
			if (threadIdx.x == 0) {
				if (k == 0) atomicMax(&ctr->sc_max_disp2_bits, v);
				else if (bounds && v) atomicMax(k < 4 ? &ctr->nb_lo[k - 1] : &ctr->nb_hi[k - 4], v);
			}
		}
	}
}

// cell size = search + 2 max|p - x|, capped (forward.cu:11818-11831)
__global__ void k_sc_setup(const StepParams* __restrict__ P, DevCounters* __restrict__ ctr)
{
	const float md2 = __uint_as_float(ctr->sc_max_disp2_bits);
	const float md = (isfinite(md2) && md2 > 0.0f) ? sqrtf(md2) : 0.0f;
	float reach = P->sc_search + 2.0f * md;
	const float cap = P->sc_search_plus16dc;
	if (reach > cap) reach = cap;
	ctr->sc_reach = reach;
	ctr->sc_inv_cell = 1.0f / reach;
}

// hash keys of start positions + bucket counts (selfColKeyKernel)
__global__ void __launch_bounds__(kBlock) k_sc_keys(int n, const float4* __restrict__ x, const DevCounters* __restrict__ ctr,
	unsigned int mask, unsigned int sentinel, unsigned int* __restrict__ keys, int* __restrict__ bucket,
	const unsigned char* __restrict__ active)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float4 p = x[i];
	const float inv_cell = ctr->sc_inv_cell;
	unsigned int k = sentinel;
	if ((!active || active[i]) && isfinite(p.x) && isfinite(p.y) && isfinite(p.z))
		k = sc_hash(sc_cell(p.x, inv_cell), sc_cell(p.y, inv_cell), sc_cell(p.z, inv_cell), mask);
	keys[i] = k;
	atomicAdd(&bucket[k], 1);
}

// exclusive scan of bucket counts, three phases (block sums, scan of sums, apply)
__global__ void __launch_bounds__(1024) k_scan_blocks(const int* __restrict__ in, int* __restrict__ out, int n,
	int* __restrict__ block_sums)
{
	__shared__ int s[1024];
	const int i = blockIdx.x * 1024 + threadIdx.x;
	const int v = (i < n) ? in[i] : 0;
	s[threadIdx.x] = v;
	__syncthreads();
	for (int o = 1; o < 1024; o <<= 1) {
		const int t = (threadIdx.x >= o) ? s[threadIdx.x - o] : 0;
		__syncthreads();
		s[threadIdx.x] += t;
		__syncthreads();
	}
	if (i < n) out[i] = s[threadIdx.x] - v;
	if (threadIdx.x == 1023) block_sums[blockIdx.x] = s[1023];
}
__global__ void __launch_bounds__(1024) k_scan_sums(int* __restrict__ sums, int nb)
{
	// single block, sequential chunks of 1024
	__shared__ int s[1024];
	__shared__ int carry;
	if (threadIdx.x == 0) carry = 0;
	__syncthreads();
	for (int base = 0; base < nb; base += 1024) {
		const int i = base + threadIdx.x;
		const int v = (i < nb) ? sums[i] : 0;
		s[threadIdx.x] = v;
		__syncthreads();
		for (int o = 1; o < 1024; o <<= 1) {
			const int t = (threadIdx.x >= o) ? s[threadIdx.x - o] : 0;
			__syncthreads();
			s[threadIdx.x] += t;
			__syncthreads();
		}
		if (i < nb) sums[i] = s[threadIdx.x] - v + carry;
		__syncthreads();
		if (threadIdx.x == 0) carry += s[1023];
		__syncthreads();
	}
}
__global__ void __launch_bounds__(1024) k_scan_add(int* __restrict__ out, int n, const int* __restrict__ sums)
{
	const int i = blockIdx.x * 1024 + threadIdx.x;
	if (i < n) out[i] += sums[blockIdx.x];
}

// scatter into buckets (unordered within a bucket)
__global__ void __launch_bounds__(kBlock) k_sc_scatter(int n, const unsigned int* __restrict__ keys,
	const int* __restrict__ start, int* __restrict__ cursor, int* __restrict__ idx_sorted)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const unsigned int k = keys[i];
	const int pos = start[k] + atomicAdd(&cursor[k], 1);
	idx_sorted[pos] = i;
}

// order each bucket by the particles' caller indices (perm maps the internal slot to
// it), which makes the counting sort equal to a stable sort of (key, caller index) —
// the reference's order; thread per bucket, insertion sort for short buckets, repeated
// minimum selection for long ones
__global__ void __launch_bounds__(kBlock) k_sc_order(int buckets, const int* __restrict__ start,
	int* __restrict__ idx_sorted, const int* __restrict__ perm)
{
	const int b = blockIdx.x * blockDim.x + threadIdx.x;
	if (b >= buckets) return;
	const int s = start[b], e = start[b + 1];
	const int len = e - s;
	if (len <= 1) return;
	if (len <= 32) {
		int v[32], key[32];
		for (int t = 0; t < len; ++t) { v[t] = idx_sorted[s + t]; key[t] = perm ? perm[v[t]] : v[t]; }
		for (int t = 1; t < len; ++t) {
			const int x = v[t], kx = key[t];
			int u = t - 1;
			while (u >= 0 && key[u] > kx) { v[u + 1] = v[u]; key[u + 1] = key[u]; --u; }
			v[u + 1] = x;
			key[u + 1] = kx;
		}
		for (int t = 0; t < len; ++t) idx_sorted[s + t] = v[t];
		return;
	}
	for (int t = 0; t < len - 1; ++t) {
		int best = t, bk = perm ? perm[idx_sorted[s + t]] : idx_sorted[s + t];
		for (int u = t + 1; u < len; ++u) {
			const int k = perm ? perm[idx_sorted[s + u]] : idx_sorted[s + u];
			if (k < bk) { bk = k; best = u; }
		}
		const int tmp = idx_sorted[s + t];
		idx_sorted[s + t] = idx_sorted[s + best];
		idx_sorted[s + best] = tmp;
	}
}

// Cell-ordered copies of what the candidate scan reads per neighbour: predicted
// position + object id, rest position + particle index, start position.  One pass,
// 48 B per particle written; the scan then reads each cell's particles contiguously.
__global__ void __launch_bounds__(kBlock) k_sc_pack(int n, const int* __restrict__ idx_sorted,
	const float4* __restrict__ X, const float4* __restrict__ Pp, const float4* __restrict__ rest,
	const int* __restrict__ obj_id, float4* __restrict__ sp, float4* __restrict__ sr, float4* __restrict__ sx)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n) return;
	const int j = idx_sorted[t];
	const float4 p = Pp[j], q = rest[j], x = X[j];
	sp[t] = make_float4(p.x, p.y, p.z, __int_as_float(j));
	sr[t] = make_float4(q.x, q.y, q.z, __int_as_float(obj_id[j]));
	sx[t] = x;
}

// The candidate list of one particle: the 27 cells around its start position in the
// reference's order (z, y, x nested, kc = 9 (z+1) + 3 (y+1) + (x+1)); a cell whose hash
// repeats an earlier one of the 27 is skipped (forward.cu:7116-7123); each cell's
// entries in bucket order through the tests of selfColBuildKernel (forward.cu:7079-7180)
// and its cap-of-32 replacement rule.  Neighbours are read from the cell-ordered copies.
// Writes contacts[i * 32 ...]; returns the count, adds the over-cap replacements to over.
__device__ __forceinline__ int sc_build_one(int i, const StepParams* __restrict__ P, const float4* __restrict__ X,
	const float4* __restrict__ Pp, const float4* __restrict__ rest, const int* __restrict__ start, unsigned int mask,
	const int* __restrict__ obj_id, const float4* __restrict__ sp, const float4* __restrict__ sr,
	const float4* __restrict__ sx, const DevCounters* __restrict__ ctr, int* __restrict__ contacts, int& over)
{
	const float4 x = X[i], p = Pp[i];
	int cnt = 0;
	if (!(isfinite(x.x) && isfinite(x.y) && isfinite(x.z) && isfinite(p.x) && isfinite(p.y) && isfinite(p.z)))
		return 0;
	const float inv_cell = ctr->sc_inv_cell;
	const float search = P->sc_search, excl2 = P->sc_excl2, cross_excl2 = P->sc_cross_excl2;
	const float fast_rel = P->sc_fast_rel;
	const int within = P->sc_within;
	// when every particle carries the same object id there are no cross-object pairs,
	// and a same-object neighbour outside the search radius is rejected right away
	const bool single_object = P->sc_single_object != 0;
	const float4 q = rest[i];
	const float dix = p.x - x.x, diy = p.y - x.y, diz = p.z - x.z;
	const int oi = obj_id[i];
	const float search2 = search * search;
	const Hash27 H(sc_cell(x.x, inv_cell), sc_cell(x.y, inv_cell), sc_cell(x.z, inv_cell), mask);
	int* out = contacts + (size_t)i * kSelfColMax;
	float prio[kSelfColMax];
	int tier[kSelfColMax];
	const unsigned int use = hash27_unique(H);
	// the used cells in order, the next cell's bucket range loaded while the current
	// cell's entries are tested
	int kc = use ? __ffs(use) - 1 : 27;
	int cs = 0, ce = 0;
	if (kc < 27) {
		const unsigned int h = H(kc);
		cs = start[h];
		ce = start[h + 1];
	}
	while (kc < 27) {
		const unsigned int later = use & ~((2u << kc) - 1u);
		const int kn = later ? __ffs(later) - 1 : 27;
		int ns = 0, ne = 0;
		if (kn < 27) {
			const unsigned int hn = H(kn);
			ns = start[hn];
			ne = start[hn + 1];
		}
		for (int t = cs; t < ce; ++t) {
			// predicted position + index first: most neighbours fail the distance
			// test, so the rest position / object id is read only for the others
			const float4 pj = sp[t];
			const int j = __float_as_int(pj.w);
			if (j == i) continue;
			const float ex = p.x - pj.x, ey = p.y - pj.y, ez = p.z - pj.z;
			const float d2 = ex * ex + ey * ey + ez * ez;
			const bool near_same = d2 < search2;
			if (!near_same && single_object) continue;
			const float4 rj = sr[t];
			const bool cross = __float_as_int(rj.w) != oi;
			if (!cross && !within) continue;
			const float qx = q.x - rj.x, qy = q.y - rj.y, qz = q.z - rj.z;
			const float q2 = qx * qx + qy * qy + qz * qz;
			float pr;
			int code = j;
			if (cross) {
				const float4 xj = sx[t];
				const float fx = x.x - xj.x, fy = x.y - xj.y, fz = x.z - xj.z;
				const float dist_x = sqrtf(fx * fx + fy * fy + fz * fz);
				const float rx = dix - (pj.x - xj.x), ry = diy - (pj.y - xj.y), rz = diz - (pj.z - xj.z);
				const float rel = sqrtf(rx * rx + ry * ry + rz * rz);
				if (!(dist_x < search + rel)) continue;
				if (!(q2 >= cross_excl2)) continue;
				pr = dist_x - rel;
				if (rel > fast_rel) code = -(j + 1);
			}
			else {
				if (!near_same) continue;
				if (!(q2 >= excl2)) continue;
				pr = sqrtf(d2);
			}
			const int tr = cross ? 0 : 1;
			if (cnt < kSelfColMax) {
				out[cnt] = code; prio[cnt] = pr; tier[cnt] = tr; ++cnt;
			}
			else {
				int worst = 0;
				for (int m = 1; m < kSelfColMax; ++m)
					if (tier[m] > tier[worst] || (tier[m] == tier[worst] && prio[m] > prio[worst])) worst = m;
				if (tr < tier[worst] || (tr == tier[worst] && pr < prio[worst])) {
					out[worst] = code; prio[worst] = pr; tier[worst] = tr;
				}
				++over;
			}
		}
		kc = kn;
		cs = ns;
		ce = ne;
	}
	return cnt;
}

// Candidate lists, one thread per particle (thread i builds particle i's list; particles
// are numbered along a Morton curve of their rest positions, so a warp's particles
// share most of their 27 cells).
__global__ void __launch_bounds__(kBlock) k_sc_build_sorted(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ X, const float4* __restrict__ Pp, const float4* __restrict__ rest,
	const int* __restrict__ idx_sorted, const int* __restrict__ start, unsigned int mask,
	const int* __restrict__ obj_id, const float4* __restrict__ sp, const float4* __restrict__ sr,
	const float4* __restrict__ sx, DevCounters* __restrict__ ctr, int* __restrict__ contacts,
	int* __restrict__ counts, const unsigned char* __restrict__ active)
{
	(void)idx_sorted;
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	int over = 0, cnt = 0;
	if (!active || active[i])
		cnt = sc_build_one(i, P, X, Pp, rest, start, mask, obj_id, sp, sr, sx, ctr, contacts, over);
	counts[i] = cnt;
	if (cnt > 0) atomicAdd(&ctr->sc_contacts, (unsigned int)cnt);
	if (over > 0) atomicAdd(&ctr->sc_overflow, (unsigned int)over);
}

// ---------------------------------------------------------------------------
// Near-pair candidate lists for a scene of one object.
//
// There every accepted pair is a same-object pair, accepted when its predicted
// positions are closer than the search radius and its rest positions at least the
// exclusion distance apart (sc_build_one's same-object branch).  The reference finds
// those pairs by scanning the 27 hashed cells around each start position (cells of
// search + 2 max|p - x|), bucket by bucket.  Here a dense grid covers the box of the
// PREDICTED positions with cells of at least kNearCellScale x search (x fastest), so a
// pair within the search radius always lies in adjacent cells, and the three cells of
// one (y, z) row around a particle are one contiguous range of the cell-sorted array:
// nine row ranges per particle instead of 27 bucket ranges (no hash, no duplicate
// buckets; longer, more even trip counts for the lanes of a warp).  The margin of the
// cell size absorbs the rounding of (p - origin) / cell.  Whatever the grid, the list
// must be the reference's: its order is the order in which the reference visits the
// pairs — the first of the particle's 27 start-position cells whose hash is the
// neighbour's bucket, then the caller index within the bucket (the stable sort) — and
// the cap-of-32 replacement rule depends on that order.  So each accepted pair gets the
// key (kc, caller index); a neighbour whose bucket is none of the 27 (possible only when
// the reference's cell size is capped) is dropped, as the reference never sees it; the
// keys are taken in ascending order in batches of kNearBatch (the batch's smallest keys
// above the last one taken, one rescan per batch) and fed through the same append /
// replacement code.  Lists, counts and the over-cap count equal the 27-cell scan's bit
// for bit.
// ---------------------------------------------------------------------------
constexpr float kNearCellScale = 1.01f;
constexpr int kNearBatch = 48;

__device__ __forceinline__ bool sc_near_member(const float4& x, const float4& p, const unsigned char* active, int i)
{
	return (!active || active[i]) && isfinite(x.x) && isfinite(x.y) && isfinite(x.z) && isfinite(p.x) &&
		isfinite(p.y) && isfinite(p.z);
}

// grid origin, cell size (>= kNearCellScale x search, grown until the cells fit `cap`)
// and cells per axis
__global__ void k_sc_near_setup(const StepParams* __restrict__ P, DevCounters* __restrict__ ctr, int cap)
{
	float cell = P->sc_search * kNearCellScale;
	float lo[3] = { 0.0f, 0.0f, 0.0f }, ext[3] = { 0.0f, 0.0f, 0.0f };
	if (ctr->nb_hi[0] | ctr->nb_hi[1] | ctr->nb_hi[2]) {
		for (int a = 0; a < 3; ++a) {
			lo[a] = f_unorder(~ctr->nb_lo[a]);
			ext[a] = fmaxf(f_unorder(ctr->nb_hi[a]) - lo[a], 0.0f);
		}
	}
	if (!(cell > 0.0f) || !isfinite(cell)) cell = 1.0f;
	double dims[3];
	for (int round = 0; round < 64; ++round) {
		double total = 1.0;
		for (int a = 0; a < 3; ++a) {
			dims[a] = floor((double)ext[a] / (double)cell) + 1.0;
			total *= dims[a];
		}
		if (total <= (double)cap) break;
		cell = (float)((double)cell * cbrt(total / (double)cap) * 1.001);
	}
	for (int a = 0; a < 3; ++a) {
		ctr->nb_origin[a] = lo[a];
		ctr->nb_dim[a] = (int)dims[a];
	}
	ctr->nb_inv = 1.0f / cell;
}

__device__ __forceinline__ int sc_near_axis(float v, float o, float inv, int dim)
{
	return min(max((int)floorf((v - o) * inv), 0), dim - 1);
}

// dense-grid keys (cell index, x fastest) of the grid's particles and cell counts;
// particles outside the reference's grid (inactive, or a start / predicted position not
// finite) are left out
__global__ void __launch_bounds__(kBlock) k_sc_near_keys(int n, const float4* __restrict__ X,
	const float4* __restrict__ Pp, const unsigned char* __restrict__ active, const DevCounters* __restrict__ ctr,
	unsigned int* __restrict__ keys, int* __restrict__ bucket)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float4 x = X[i], p = Pp[i];
	unsigned int k = 0xffffffffu;
	if (sc_near_member(x, p, active, i)) {
		const float inv = ctr->nb_inv;
		const int dx = ctr->nb_dim[0], dy = ctr->nb_dim[1], dz = ctr->nb_dim[2];
		const int ix = sc_near_axis(p.x, ctr->nb_origin[0], inv, dx);
		const int iy = sc_near_axis(p.y, ctr->nb_origin[1], inv, dy);
		const int iz = sc_near_axis(p.z, ctr->nb_origin[2], inv, dz);
		k = (unsigned int)((iz * dy + iy) * dx + ix);
		atomicAdd(&bucket[k], 1);
	}
	keys[i] = k;
}

// scatter predicted position + index into the cells (order within a cell is free: the
// lists are ordered by key afterwards); leaves the cell counts at zero; a particle outside
// the grid gets its empty candidate list here
__global__ void __launch_bounds__(kBlock) k_sc_near_scatter(int n, const unsigned int* __restrict__ keys,
	const int* __restrict__ start, int* __restrict__ bucket, const float4* __restrict__ Pp, float4* __restrict__ fp,
	int* __restrict__ counts)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const unsigned int k = keys[i];
	if (k == 0xffffffffu) { counts[i] = 0; return; }
	const int pos = start[k] + atomicSub(&bucket[k], 1) - 1;
	const float4 p = Pp[i];
	fp[pos] = make_float4(p.x, p.y, p.z, __int_as_float(i));
}

// the key of accepted neighbour j of particle i: the first of i's 27 start cells
// (reference order) whose hash is j's bucket, then j's caller index; ~0 = never visited
__device__ __forceinline__ unsigned long long sc_near_key(const Hash27& Href, float4 xj, float inv_cell,
	unsigned int caller_j)
{
	const unsigned int hj =
		sc_hash(sc_cell(xj.x, inv_cell), sc_cell(xj.y, inv_cell), sc_cell(xj.z, inv_cell), Href.mask);
	for (int kc = 0; kc < 27; ++kc)
		if (Href(kc) == hj) return ((unsigned long long)kc << 32) | caller_j;
	return ~0ull;
}

// mask: the reference's hash table mask (for the keys); start_f / fp: the dense grid's
// cell starts and (p, index) by cell.  Thread t takes the t-th particle in cell order, so
// the lanes of a warp share cells and row ranges and run even trip counts (particles
// outside the grid got their zero count from k_sc_near_scatter).
// six resident blocks per SM: the row scans are latency bound; the spills fall in the
// rarely used key batches
__global__ void __launch_bounds__(kBlock, 6) k_sc_build_near(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ X, const float4* __restrict__ Pp, const float4* __restrict__ rest,
	const unsigned char* __restrict__ active, const int* __restrict__ start_f, unsigned int mask,
	const float4* __restrict__ fp, const int* __restrict__ perm, DevCounters* __restrict__ ctr,
	int* __restrict__ contacts, int* __restrict__ counts)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= start_f[ctr->nb_dim[0] * ctr->nb_dim[1] * ctr->nb_dim[2]]) return;
	const int i = __float_as_int(fp[t].w);
	int cnt = 0, over = 0;
	const float4 x = X[i], p = Pp[i];
	if (P->sc_within) {
		const float search = P->sc_search, excl2 = P->sc_excl2;
		const float search2 = search * search;
		const float4 q = rest[i];
		const float inv = ctr->nb_inv;
		const int dx = ctr->nb_dim[0], dy = ctr->nb_dim[1], dz = ctr->nb_dim[2];
		const int ix = sc_near_axis(p.x, ctr->nb_origin[0], inv, dx);
		const int iy = sc_near_axis(p.y, ctr->nb_origin[1], inv, dy);
		const int iz = sc_near_axis(p.z, ctr->nb_origin[2], inv, dz);
		const int x0 = max(ix - 1, 0), x1 = min(ix + 1, dx - 1);
		// row r = 3 (dz + 1) + (dy + 1): its cells x0..x1 are one range of the sorted array
		auto row_range = [&](int r, int& cs, int& ce) {
			const int qr = (r * 11) >> 5;   // r / 3
			const int z = iz + qr - 1, y = iy + (r - 3 * qr) - 1;
			cs = ce = 0;
			if (z >= 0 && z < dz && y >= 0 && y < dy) {
				const int row = (z * dy + y) * dx;
				cs = start_f[row + x0];
				ce = start_f[row + x1 + 1];
			}
		};
		// the particle's own reference cell, for the keys
		const float inv_cell = ctr->sc_inv_cell;
		const Hash27 Href(sc_cell(x.x, inv_cell), sc_cell(x.y, inv_cell), sc_cell(x.z, inv_cell), mask);
		int* out = contacts + (size_t)i * kSelfColMax;
		float prio[kSelfColMax];
		int tier[kSelfColMax];
		unsigned long long last = 0ull;
		bool first_batch = true;
		for (;;) {
			// the kNearBatch smallest keys above `last`, ascending
			unsigned long long bk[kNearBatch];
			float bd2[kNearBatch];
			int bj[kNearBatch];
			int nb = 0;
			bool more = false;
			// the nine rows in turn, the next row's range loaded while the current one's
			// entries are tested
			int cs, ce;
			row_range(0, cs, ce);
			for (int r = 0; r < 9; ++r) {
				int ns = 0, ne = 0;
				if (r < 8) row_range(r + 1, ns, ne);
				for (int t = cs; t < ce; ++t) {
					const float4 pj = fp[t];
					const int j = __float_as_int(pj.w);
					if (j == i) continue;
					const float ex = p.x - pj.x, ey = p.y - pj.y, ez = p.z - pj.z;
					const float d2 = ex * ex + ey * ey + ez * ez;
					if (!(d2 < search2)) continue;
					const float4 rj = rest[j];
					const float qx = q.x - rj.x, qy = q.y - rj.y, qz = q.z - rj.z;
					const float q2 = qx * qx + qy * qy + qz * qz;
					if (!(q2 >= excl2)) continue;
					const unsigned long long key =
						sc_near_key(Href, X[j], inv_cell, (unsigned int)(perm ? perm[j] : j));
					if (key == ~0ull || (!first_batch && key <= last)) continue;
					if (nb == kNearBatch) {
						more = true;
						if (key >= bk[kNearBatch - 1]) continue;
						--nb;   // the largest leaves the batch
					}
					int m = nb;
					while (m > 0 && bk[m - 1] > key) {
						bk[m] = bk[m - 1]; bd2[m] = bd2[m - 1]; bj[m] = bj[m - 1];
						--m;
					}
					bk[m] = key; bd2[m] = d2; bj[m] = j;
					++nb;
				}
				cs = ns;
				ce = ne;
			}
			// the reference's append / replacement, in key order
			for (int a = 0; a < nb; ++a) {
				const float pr = sqrtf(bd2[a]);
				const int tr = 1;
				if (cnt < kSelfColMax) {
					out[cnt] = bj[a]; prio[cnt] = pr; tier[cnt] = tr; ++cnt;
				}
				else {
					int worst = 0;
					for (int m = 1; m < kSelfColMax; ++m)
						if (tier[m] > tier[worst] || (tier[m] == tier[worst] && prio[m] > prio[worst])) worst = m;
					if (tr < tier[worst] || (tr == tier[worst] && pr < prio[worst])) {
						out[worst] = bj[a]; prio[worst] = pr; tier[worst] = tr;
					}
					++over;
				}
			}
			if (!more) break;
			last = bk[nb - 1];
			first_batch = false;
		}
	}
	counts[i] = cnt;
	if (cnt > 0) atomicAdd(&ctr->sc_contacts, (unsigned int)cnt);
	if (over > 0) atomicAdd(&ctr->sc_overflow, (unsigned int)over);
}

__device__ __forceinline__ bool sc_start_normal(float4 xi, float4 xj, float4 qi, float4 qj, float& nx, float& ny,
	float& nz)
{
	nx = xi.x - xj.x; ny = xi.y - xj.y; nz = xi.z - xj.z;
	float l2 = nx * nx + ny * ny + nz * nz;
	if (!(l2 > 1e-24f)) {
		nx = qi.x - qj.x; ny = qi.y - qj.y; nz = qi.z - qj.z;
		l2 = nx * nx + ny * ny + nz * nz;
		if (!(l2 > 1e-24f)) return false;
	}
	const float inv = 1.0f / sqrtf(l2);
	nx *= inv; ny *= inv; nz *= inv;
	return true;
}

// phase 1 of the per-iteration contact projection (selfColSolveKernel, forward.cu:7205-7308)
// eight resident blocks per SM: 0.58 -> 0.50 ms per frame at 1M (the same bound made
// the collider projection slower: 0.75 -> 0.83)
__global__ void __launch_bounds__(kBlock, 8) k_sc_solve(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ pos, const float4* __restrict__ pos_start, const float4* __restrict__ rest,
	const int* __restrict__ contacts, const int* __restrict__ counts, const DevCounters* __restrict__ ctr,
	float4* __restrict__ dp_out, float4* __restrict__ dp_cross)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	if (ctr->sc_contacts == 0u) return;
	const int cnt = counts[i];
	if (cnt <= 0) return;
	const float dc = P->sc_dc;
	const float ims = P->inv_mass_scale;
	const float4 pi = pos[i];
	const float wi = pi.w * ims;
	float ax = 0.0f, ay = 0.0f, az = 0.0f;
	int act = 0;
	float cpx = 0.0f, cpy = 0.0f, cpz = 0.0f;
	float sx = 0.0f, sy = 0.0f, sz = 0.0f, w_fast = 0.0f;
	int n_fast = 0;
	const int* list = contacts + (size_t)i * kSelfColMax;
	const float4 xi = pos_start[i], qi = rest[i];
	if (wi > 0.0f) {
		const float dc2 = dc * dc;
		for (int k = 0; k < cnt; ++k) {
			const int code = list[k];
			if (code < 0) {
				const int j = -code - 1;
				float nx, ny, nz;
				if (!sc_start_normal(xi, pos_start[j], qi, rest[j], nx, ny, nz)) continue;
				const float4 pj = pos[j];
				const float proj = (pi.x - pj.x) * nx + (pi.y - pj.y) * ny + (pi.z - pj.z) * nz;
				if (!(proj < dc)) continue;
				const float pen = dc - proj;
				sx += nx * pen; sy += ny * pen; sz += nz * pen;
				const float wj = pj.w * ims;
				w_fast += wi / (wi + wj);
				++n_fast;
				continue;
			}
			const int j = code;
			const float4 pj = pos[j];
			const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
			const float d2 = dx * dx + dy * dy + dz * dz;
			if (!(d2 < dc2)) continue;
			const float wj = pj.w * ims;
			const float wr = wi / (wi + wj);
			if (d2 < 1e-24f) {
				const float4 qj = rest[j];
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
	float3 out = (act > 0) ? make_float3(ax / act, ay / act, az / act) : make_float3(0.0f, 0.0f, 0.0f);
	if (n_fast > 0) {
		const float sl = sqrtf(sx * sx + sy * sy + sz * sz);
		if (sl > 1e-20f) {
			const float bx = sx / sl, by = sy / sl, bz = sz / sl;
			float delta = 0.0f;
			for (int k = 0; k < cnt; ++k) {
				const int code = list[k];
				if (code >= 0) continue;
				const int j = -code - 1;
				float nx, ny, nz;
				if (!sc_start_normal(xi, pos_start[j], qi, rest[j], nx, ny, nz)) continue;
				const float4 pj = pos[j];
				const float ddx = pi.x - pj.x, ddy = pi.y - pj.y, ddz = pi.z - pj.z;
				if (!(ddx * nx + ddy * ny + ddz * nz < dc)) continue;
				const float pen = dc - (ddx * bx + ddy * by + ddz * bz);
				if (pen > delta) delta = pen;
			}
			if (delta > 0.0f) {
				const float sc = delta * (w_fast / (float)n_fast);
				cpx = bx * sc; cpy = by * sc; cpz = bz * sc;
				out = make_float3(out.x + cpx, out.y + cpy, out.z + cpz);
			}
		}
	}
	dp_out[i] = make_float4(out.x, out.y, out.z, 0.0f);
	if (dp_cross) dp_cross[i] = make_float4(cpx, cpy, cpz, 0.0f);
}

// ---------------------------------------------------------------------------
// pins (attachApplyKernel, forward.cu:6714-6725): inverse mass 0, position, zero velocity
// ---------------------------------------------------------------------------
__global__ void k_attach(int count, const int* __restrict__ idx, const float* __restrict__ pos, int n,
	float4* __restrict__ pos_curr, float4* __restrict__ vel, float* __restrict__ obj_w, float weight)
{
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= count) return;
	const int i = idx[k];
	if (i < 0 || i >= n) return;
	pos_curr[i] = make_float4(pos[3 * k], pos[3 * k + 1], pos[3 * k + 2], 0.0f);
	vel[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	if (obj_w) obj_w[i] = weight;   // rigid-fit weight of object mode (forward.cu:6724)
}

// caller-order positions into the internal order, inverse masses kept
__global__ void k_set_positions(int n, const float* __restrict__ pos3, const int* __restrict__ perm,
	float4* __restrict__ pos, float* __restrict__ pos_out3)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int o = perm[i];
	const float x = pos3[3 * o], y = pos3[3 * o + 1], z = pos3[3 * o + 2];
	pos[i] = make_float4(x, y, z, pos[i].w);
	pos_out3[3 * o] = x; pos_out3[3 * o + 1] = y; pos_out3[3 * o + 2] = z;
}

// serving arena: copy of an index array with every non-negative entry shifted by delta
__global__ void k_copy_shift(long long count, const int* __restrict__ src, int* __restrict__ dst, int delta)
{
	const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= count) return;
	const int v = src[i];
	dst[i] = v >= 0 ? v + delta : v;
}
__global__ void k_fill_int(int n, int* __restrict__ a, int v)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) a[i] = v;
}
// a retired session's rows stay in place, frozen: inverse mass 0 (also the value pin
// releases restore), velocity 0
__global__ void k_freeze_rows(int n, float4* __restrict__ pos, float4* __restrict__ vel, float* __restrict__ saved_w)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	pos[i].w = 0.0f;
	vel[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	saved_w[i] = 0.0f;
}

__global__ void k_fill(int n, float* __restrict__ a, float v)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) a[i] = v;
}

__global__ void k_get_w(int n, const float4* __restrict__ pos, float* __restrict__ w)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) w[i] = pos[i].w;
}
__global__ void k_set_w(int n, float4* __restrict__ pos, const float* __restrict__ w, float value)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) pos[i].w = w ? w[i] : value;
}

// addRigidVelocityAllKernel (forward.cu:6701-6712)
__global__ void k_add_rigid_velocity(int n, const float4* __restrict__ pos, float4* __restrict__ vel, float3 dv,
	float3 dw, float3 c)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float4 p = pos[i];
	if (p.w <= 0.0f) return;
	const float rx = p.x - c.x, ry = p.y - c.y, rz = p.z - c.z;
	const float4 v = vel[i];
	vel[i] = make_float4(v.x + dv.x + (dw.y * rz - dw.z * ry), v.y + dv.y + (dw.z * rx - dw.x * rz),
		v.z + dv.z + (dw.x * ry - dw.y * rx), 0.0f);
}

// ---------------------------------------------------------------------------
// volume-weighted J statistics (computeVolumeJKernel forward.cu:9428-9476 + the
// host reduction forward.cu:12670-12689), reduced on the device in double
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) k_jstats(int n, const float4* __restrict__ pos, const int* __restrict__ voff,
	const int* __restrict__ vidx, const float* __restrict__ det_rest, const int* __restrict__ mat_type,
	const float* __restrict__ v_rest, DevCounters* __restrict__ ctr)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	double a = 0.0, b = 0.0, c2 = 0.0;
	if (idx < n && mat_type[idx] == 0) {
		float J = 1.0f;
		const int off = voff[idx], cnt = voff[idx + 1] - off;
		float3 c = f3(pos[idx]);
		int used = 0;
		for (int k = 0; k < cnt; ++k) {
			const int j = vidx[off + k];
			if (j < 0 || j >= n) continue;
			c = add3(c, f3(pos[j]));
			++used;
		}
		if (used >= 3) {
			const float inv_n = 1.0f / (float)(used + 1);
			c = mul3(c, inv_n);
			M3 S;
			m3_zero(S);
			{
				const float3 d = sub3(f3(pos[idx]), c);
				m3_add_outer(S, d, d);
			}
			for (int k = 0; k < cnt; ++k) {
				const int j = vidx[off + k];
				if (j < 0 || j >= n) continue;
				const float3 d = sub3(f3(pos[j]), c);
				m3_add_outer(S, d, d);
			}
			for (int cc = 0; cc < 3; ++cc)
				for (int r = 0; r < 3; ++r) S.m[cc][r] *= inv_n;
			float s_cur, det_hat;
			if (sigma_scale_det(S, s_cur, det_hat)) {
				const float det_cur = s_cur * s_cur * s_cur * det_hat;
				const float dr = det_rest[idx];
				if (!(dr < 1e-30f)) {
					const float Jc = sqrtf(det_cur / dr);
					if (isfinite(Jc) && Jc > 0.0f) J = Jc;
				}
			}
		}
		const double v = (double)v_rest[idx];
		if (v > 0.0 && isfinite(v)) { a = v; b = v * J; c2 = v * (double)J * J; }
	}
	for (int o = 16; o > 0; o >>= 1) {
		a += __shfl_xor_sync(0xffffffffu, a, o);
		b += __shfl_xor_sync(0xffffffffu, b, o);
		c2 += __shfl_xor_sync(0xffffffffu, c2, o);
	}
	if ((threadIdx.x & 31) == 0 && (a != 0.0 || b != 0.0)) {
		atomicAdd(&ctr->jstats[0], a);
		atomicAdd(&ctr->jstats[1], b);
		atomicAdd(&ctr->jstats[2], c2);
	}
}

// ---------------------------------------------------------------------------
// deformed Gaussian shapes (deformedShapeKernel, forward.cu:13063-13225; robust
// F estimate forward.cu:450) with the FP64 Jacobi of symEig3Double (13022-13060)
// ---------------------------------------------------------------------------
// Eigen-decomposition of a symmetric 3x3 matrix in FP64 by cyclic Jacobi sweeps over the
// pivots (0,1), (0,2), (1,2) (symEig3Double's order and stop: off-diagonal mass below
// 1e-15 of the diagonal's, at most 32 sweeps), each rotation the one shape matching uses
// (jacobi_rotate_d).  Columns of V: eigenvectors; ev: eigenvalues in diagonal order.
__device__ __noinline__ void sym_eig3_double(double (&a)[3][3], double (&ev)[3], double (&V)[3][3])
{
#pragma unroll
	for (int r = 0; r < 3; ++r)
#pragma unroll
		for (int c = 0; c < 3; ++c) V[r][c] = (r == c) ? 1.0 : 0.0;
	for (int sweep = 0; sweep < 32; ++sweep) {
		const double off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
		const double diag = fabs(a[0][0]) + fabs(a[1][1]) + fabs(a[2][2]);
		if (off <= 1e-15 * diag + 1e-300) break;
		if (fabs(a[0][1]) > 1e-300) jacobi_rotate_d<0, 1>(a, V);
		if (fabs(a[0][2]) > 1e-300) jacobi_rotate_d<0, 2>(a, V);
		if (fabs(a[1][2]) > 1e-300) jacobi_rotate_d<1, 2>(a, V);
	}
	ev[0] = a[0][0]; ev[1] = a[1][1]; ev[2] = a[2][2];
}

__global__ void __launch_bounds__(kBlock) k_deformed_shapes(int n, const float4* __restrict__ rest,
	const float4* __restrict__ cur, const int* __restrict__ off, const int* __restrict__ nbr,
	const float* __restrict__ scales, const float* __restrict__ rots, float deform_eps, float* __restrict__ out_scale,
	float* __restrict__ out_quat, DevCounters* __restrict__ ctr, const int* __restrict__ perm)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int o = perm ? perm[i] : i;   // output slot in the caller's order
	const float3 s0 = make_float3(scales[3 * i], scales[3 * i + 1], scales[3 * i + 2]);
	const float4 q0 = make_float4(rots[4 * i], rots[4 * i + 1], rots[4 * i + 2], rots[4 * i + 3]);
	const float3 x = f3(cur[i]), x0 = f3(rest[i]);
	const float dxv = x.x - x0.x, dyv = x.y - x0.y, dzv = x.z - x0.z;
	const float diff = sqrtf(dxv * dxv + dyv * dyv + dzv * dzv);
	const int e0 = off[i], kn = off[i + 1] - e0;
	bool deformed = false;
	M3 Sigma;
	m3_zero(Sigma);
	if (diff > deform_eps && kn >= 3) {
		M3 PPt, QPt;
		m3_zero(PPt);
		m3_zero(QPt);
		for (int k = 0; k < kn; ++k) {
			const int j = nbr[e0 + k];
			if (j < 0 || j >= n) continue;
			const float4 rj = rest[j], cj = cur[j];
			const float3 p = make_float3(rj.x - x0.x, rj.y - x0.y, rj.z - x0.z);
			const float3 q = make_float3(cj.x - x.x, cj.y - x.y, cj.z - x.z);
			m3_add_outer(PPt, p, p);
			m3_add_outer(QPt, q, p);
		}
		const float tr_p = PPt.m[0][0] + PPt.m[1][1] + PPt.m[2][2];
		const float alpha = (tr_p > 0.0f) ? (tr_p * 1e-4f) : 1e-6f;
#pragma unroll
		for (int d = 0; d < 3; ++d) { PPt.m[d][d] = PPt.m[d][d] + alpha; QPt.m[d][d] = QPt.m[d][d] + alpha; }
		const float sp = fmaxf((PPt.m[0][0] + PPt.m[1][1] + PPt.m[2][2]) * (1.0f / 3.0f), 1e-30f);
		const float inv_sp = 1.0f / sp;
		M3 Ph, inv_hat;
#pragma unroll
		for (int c = 0; c < 3; ++c)
#pragma unroll
			for (int r = 0; r < 3; ++r) Ph.m[c][r] = PPt.m[c][r] * inv_sp;
		if (inverse3x3_safe(Ph, inv_hat, 1e-9f)) {
			M3 inv_p;
#pragma unroll
			for (int c = 0; c < 3; ++c)
#pragma unroll
				for (int r = 0; r < 3; ++r) inv_p.m[c][r] = inv_hat.m[c][r] * inv_sp;
			const M3 A = m3_mul(QPt, inv_p);
			const M3 AtA = m3_mul(m3_t(A), A);
			M3 V;
			float3 S2;
			eig_sym3f(AtA, S2, V);
			float3 Sv = make_float3(sqrtf(fmaxf(0.0f, S2.x)), sqrtf(fmaxf(0.0f, S2.y)), sqrtf(fmaxf(0.0f, S2.z)));
			Sv = make_float3(fminf(fmaxf(Sv.x, 1e-3f), 1.5f), fminf(fmaxf(Sv.y, 1e-3f), 1.5f), fminf(fmaxf(Sv.z, 1e-3f), 1.5f));
			M3 Si;
			m3_zero(Si);
			Si.m[0][0] = (Sv.x > 1.0e-7f) ? 1.0f / Sv.x : 0.0f;
			Si.m[1][1] = (Sv.y > 1.0e-7f) ? 1.0f / Sv.y : 0.0f;
			Si.m[2][2] = (Sv.z > 1.0e-7f) ? 1.0f / Sv.z : 0.0f;
			M3 U = m3_mul(m3_mul(A, V), Si);
			const M3 Vt = m3_t(V);
			M3 R = m3_mul(U, Vt);
			if (m3_det(R) < 0.0f) {
				U.m[0][0] *= -1.0f; U.m[0][1] *= -1.0f; U.m[0][2] *= -1.0f;
				R = m3_mul(U, Vt);
			}
			M3 Sd;
			m3_zero(Sd);
			Sd.m[0][0] = Sv.x; Sd.m[1][1] = Sv.y; Sd.m[2][2] = Sv.z;
			const M3 S_final = m3_mul(m3_mul(V, Sd), Vt);
			M3 Sm;
			m3_zero(Sm);
			Sm.m[0][0] = s0.x; Sm.m[1][1] = s0.y; Sm.m[2][2] = s0.z;
			const float r = q0.x, qx = q0.y, qy = q0.z, qz = q0.w;
			M3 R0;
			R0.m[0][0] = 1.f - 2.f * (qy * qy + qz * qz); R0.m[0][1] = 2.f * (qx * qy - r * qz);
			R0.m[0][2] = 2.f * (qx * qz + r * qy);
			R0.m[1][0] = 2.f * (qx * qy + r * qz); R0.m[1][1] = 1.f - 2.f * (qx * qx + qz * qz);
			R0.m[1][2] = 2.f * (qy * qz - r * qx);
			R0.m[2][0] = 2.f * (qx * qz - r * qy); R0.m[2][1] = 2.f * (qy * qz + r * qx);
			R0.m[2][2] = 1.f - 2.f * (qx * qx + qy * qy);
			const M3 M = m3_mul(m3_mul(m3_mul(Sm, R0), S_final), m3_t(R));
			Sigma = m3_mul(m3_t(M), M);
			deformed = m3_finite(Sigma);
		}
	}
	const double tr = deformed ? ((double)Sigma.m[0][0] + Sigma.m[1][1] + Sigma.m[2][2]) : 0.0;
	if (!deformed || !(tr > 0.0)) {
		out_scale[3 * o + 0] = s0.x; out_scale[3 * o + 1] = s0.y; out_scale[3 * o + 2] = s0.z;
		out_quat[4 * o + 0] = q0.x; out_quat[4 * o + 1] = q0.y; out_quat[4 * o + 2] = q0.z; out_quat[4 * o + 3] = q0.w;
		atomicAdd(&ctr->shapes_kept, 1u);
		return;
	}
	const double inv = 3.0 / tr;
	double a[3][3];
#pragma unroll
	for (int rr = 0; rr < 3; ++rr)
#pragma unroll
		for (int c = 0; c < 3; ++c) a[rr][c] = 0.5 * ((double)Sigma.m[c][rr] + (double)Sigma.m[rr][c]) * inv;
	double ev[3], E[3][3];
	sym_eig3_double(a, ev, E);
	const double det = E[0][0] * (E[1][1] * E[2][2] - E[1][2] * E[2][1])
		- E[0][1] * (E[1][0] * E[2][2] - E[1][2] * E[2][0])
		+ E[0][2] * (E[1][0] * E[2][1] - E[1][1] * E[2][0]);
	if (det < 0.0) {
#pragma unroll
		for (int rr = 0; rr < 3; ++rr) E[rr][2] = -E[rr][2];
	}
	const double s_floor = 1e-3 * (double)fmaxf(s0.x, fmaxf(s0.y, s0.z));
#pragma unroll
	for (int k = 0; k < 3; ++k) out_scale[3 * o + k] = (float)fmax(sqrt(fmax(ev[k], 0.0) / inv), s_floor);
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
	out_quat[4 * o + 0] = (float)(w / qn);
	out_quat[4 * o + 1] = (float)(qxv / qn);
	out_quat[4 * o + 2] = (float)(qyv / qn);
	out_quat[4 * o + 3] = (float)(qzv / qn);
	atomicAdd(&ctr->shapes_deformed, 1u);
}

// ===========================================================================
// The whole substep in one cooperative launch: predict, then per iteration distance,
// volume solve and gather, shape matching and the projections, then the velocity
// commit, with a grid-wide barrier between phases.  Every phase runs the same
// per-item code as its own kernel (the *_row / *_lane functions above, with plain
// loads for the data the launch itself writes), so the result is that of the kernel
// sequence bit for bit; what changes is one launch per substep instead of one per
// phase.  Covers the default forms (Jacobi distance, 4-lane one-pass volume solve and
// gather, shape matching, colliders, ground, press, contact shapes); self-collision,
// object mode and the Gauss-Seidel forms keep the kernel sequence.
// ===========================================================================
struct SubstepArgs {
	int n, iters, use_distance, use_volume, use_shape, shape_robust, project;
	const StepParams* P;
	float4 *pos_curr, *pos_next, *pos_tmp, *vel;
	float* lam_vol;
	const float4* cshape;
	const float* crmax;
	float* crg;
	const int *off, *nbr;
	const float *ndist, *nstiff;
	float* lam;
	const int *vol_off, *vol_idx, *mat_type, *rev_off, *rev_idx;
	const float *det_rest, *rest_len;
	float4* rec;
	float* recz;
	const float4 *pos_rest, *shape_rest;
	float4* shape_q;
	DevCounters* ctr;
	const int* obj_id;
	const KinCollider* ext_kin;
	const int2* ext_range;
	float* pos_out3;
	const int* perm;
};

// Grid-wide barrier of the fused launch (all blocks are co-resident: the launch is
// cooperative).  Thread 0 of each block publishes its block's writes, arrives, and the
// last to arrive opens the next generation; the wait is bounded (about 2^24 polls of at
// least 64 ns): if it runs out, bar_timeout is set and the launch runs to its end with
// the host reporting the error, instead of hanging the GPU.
__device__ __forceinline__ void grid_barrier(DevCounters* __restrict__ ctr)
{
	__syncthreads();
	if (threadIdx.x == 0) {
		volatile unsigned int* gen = &ctr->bar_gen;
		const unsigned int g = *gen;
		__threadfence();
		if (atomicAdd(&ctr->bar_count, 1u) + 1u == gridDim.x) {
			ctr->bar_count = 0u;
			__threadfence();
			atomicAdd(&ctr->bar_gen, 1u);
		}
		else {
			unsigned int polls = 0;
			while (*gen == g) {
				if (++polls > (1u << 24)) { atomicExch(&ctr->bar_timeout, 1u); break; }
				__nanosleep(64);
			}
		}
		__threadfence();
	}
	__syncthreads();
}

__global__ void __launch_bounds__(kBlock, 2) k_substep_fused(SubstepArgs A)
{
	DevCounters* ctr = A.ctr;
	const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	const long long nth = (long long)gridDim.x * blockDim.x;
	const int lane = threadIdx.x & 31;
	const long long wbase = tid - lane;   // lane-group phases: whole warps iterate together
	const int n = A.n;
	const StepParams* P = A.P;
	for (long long i = tid; i < n; i += nth)
		predict_row((int)i, n, P, A.pos_curr, A.pos_next, A.vel, A.use_volume ? A.lam_vol : nullptr, A.cshape, A.crg);
	grid_barrier(ctr);
	float4* pin = A.pos_next;
	float4* pout = A.pos_tmp;
	for (int it = 0; it < A.iters; ++it) {
		const int first = (it == 0), last = (it == A.iters - 1);
		if (A.use_distance) {
			for (long long i = tid; i < n; i += nth)
				distance_row<false>((int)i, n, P, pin, pout, A.off, A.nbr, A.ndist, A.nstiff, A.lam, first ? 0 : 1,
					last ? 0 : 1);
			grid_barrier(ctr);
			float4* t = pin; pin = pout; pout = t;
		}
		if (A.use_volume) {
			for (long long b = wbase; b < 4LL * n; b += nth)
				solve_onepass_lane<4, false>(b + lane, n, P, pin, A.vol_off, A.vol_idx, A.det_rest, A.mat_type, A.lam_vol,
					A.rec, A.recz, first ? 0 : 1);
			grid_barrier(ctr);
			for (long long b = wbase; b < 4LL * n; b += nth)
				gather_group_lane<4, false>(b + lane, n, P, pin, pout, A.rev_off, A.rev_idx, A.rec, A.recz, A.rest_len);
			grid_barrier(ctr);
			float4* t = pin; pin = pout; pout = t;
		}
		if (A.use_shape) {
			for (long long i = tid; i < n; i += nth) {
				if (A.shape_robust)
					shape_row<true, false>((int)i, n, P, pin, pout, A.pos_rest, A.off, A.nbr, A.shape_rest, A.shape_q);
				else
					shape_row<false, false>((int)i, n, P, pin, pout, A.pos_rest, A.off, A.nbr, A.shape_rest, A.shape_q);
			}
			grid_barrier(ctr);
			float4* t = pin; pin = pout; pout = t;
		}
		if (A.project) {
			for (long long i = tid; i < n; i += nth)
				project_row((int)i, n, P, pin, A.pos_curr, nullptr, nullptr, A.ctr, last ? 1 : 0, A.obj_id, A.ext_kin,
					A.ext_range, nullptr, nullptr, A.cshape, A.crmax, A.crg);
			grid_barrier(ctr);
		}
	}
	for (long long i = tid; i < n; i += nth) velocity_row((int)i, n, P, A.pos_curr, pin, A.vel, A.pos_out3, A.perm, A.crg);
}

// ===========================================================================
// Upload-time cluster builder on the GPU (every Gaussian a leader): k-ring BFS and the
// farthest-point subsample of rebuildVolumeClusters (forward.cu:9814-10033), one warp
// per leader, in the caller's index space.  Same visiting order, same candidate order,
// same float distances (explicit roundings, as the host computes them) and the same
// first-maximum ties as the host builder, so the member lists are identical.  A leader
// whose ball exceeds kBallCap candidates is flagged and built on the host.
// ===========================================================================
constexpr int kBallCap = 1024;        // BFS candidates a warp holds
constexpr int kBallSet = 2048;        // visited-set slots (open addressing, power of two)
constexpr int kBuildWarps = 4;        // warps per block
constexpr size_t kBuildSmem = (size_t)kBuildWarps * (kBallCap * 8 + kBallSet * 4);

__device__ __forceinline__ float build_dist2(const float* __restrict__ a, const float* __restrict__ b)
{
	const float dx = __fsub_rn(a[0], b[0]), dy = __fsub_rn(a[1], b[1]), dz = __fsub_rn(a[2], b[2]);
	return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

__device__ __forceinline__ unsigned int build_slot(int j) { return ((unsigned int)j * 2654435761u) & (kBallSet - 1); }

__device__ __forceinline__ bool build_set_has(const int* set, int j)
{
	for (unsigned int h = build_slot(j), t = 0; t < kBallSet; ++t, h = (h + 1) & (kBallSet - 1)) {
		const int v = set[h];
		if (v == j) return true;
		if (v == -1) return false;
	}
	return false;
}

__device__ __forceinline__ void build_set_put(int* set, int j)
{
	for (unsigned int h = build_slot(j), t = 0; t < kBallSet; ++t, h = (h + 1) & (kBallSet - 1)) {
		const int old = atomicCAS(&set[h], -1, j);
		if (old == -1 || old == j) return;
	}
}

// warp-wide (value, index) maximum, lowest index among equal values
__device__ __forceinline__ void build_argmax(float& v, int& m)
{
	for (int o = 16; o > 0; o >>= 1) {
		const float v2 = __shfl_xor_sync(0xffffffffu, v, o);
		const int m2 = __shfl_xor_sync(0xffffffffu, m, o);
		if (v2 > v || (v2 == v && m2 >= 0 && (m < 0 || m2 < m))) { v = v2; m = m2; }
	}
}

__global__ void __launch_bounds__(kBuildWarps * 32) k_build_members(int n, int first, int last,
	const int* __restrict__ off, const int* __restrict__ nbr, const float* __restrict__ rest3, int ring_k, int cap,
	int* __restrict__ members, int* __restrict__ counts)
{
	// lists of nodes [first, last); node i's at members[(i - first) * cap ...], counts[i - first]
	extern __shared__ int build_sm[];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
	int* col = build_sm + w * (kBallCap * 2 + kBallSet);
	float* md = reinterpret_cast<float*>(col + kBallCap);
	int* set = col + 2 * kBallCap;
	const unsigned int lt = (1u << lane) - 1u;
	for (int i = first + blockIdx.x * kBuildWarps + w; i < last; i += gridDim.x * kBuildWarps) {
		int count = 0;
		bool overflow = false;
		if (ring_k <= 1) {
			for (int e0 = off[i]; e0 < off[i + 1] && !overflow; e0 += 32) {
				const int e = e0 + lane;
				int j = -1;
				if (e < off[i + 1]) j = nbr[e];
				const bool ok = j >= 0 && j < n && j != i;
				const unsigned int m = __ballot_sync(0xffffffffu, ok);
				const int pos = count + __popc(m & lt);
				if (ok && pos < kBallCap) col[pos] = j;
				count += __popc(m);
				if (count > kBallCap) overflow = true;
			}
		}
		else {
			for (int t = lane; t < kBallSet; t += 32) set[t] = -1;
			__syncwarp();
			if (lane == 0) build_set_put(set, i);
			__syncwarp();
			int fs = 0, fe = 0;          // frontier = col[fs, fe); the leader alone at depth 0
			for (int d = 0; d < ring_k && !overflow; ++d) {
				if (d > 0 && fs == fe) break;
				const int next = count;
				const int nf = (d == 0) ? 1 : fe - fs;
				for (int q = 0; q < nf && !overflow; ++q) {
					const int f = (d == 0) ? i : col[fs + q];
					const int r1 = off[f + 1];
					for (int e0 = off[f]; e0 < r1 && !overflow; e0 += 32) {
						const int e = e0 + lane;
						int j = -1;
						if (e < r1) j = nbr[e];
						bool fresh = j >= 0 && j < n;
						// repeated entries in one row: only the first lane's counts
						const unsigned int same = __match_any_sync(0xffffffffu, j);
						if ((same & lt) != 0u) fresh = false;
						if (fresh && build_set_has(set, j)) fresh = false;
						const unsigned int m = __ballot_sync(0xffffffffu, fresh);
						const int pos = count + __popc(m & lt);
						if (fresh && pos < kBallCap) { col[pos] = j; build_set_put(set, j); }
						count += __popc(m);
						if (count > kBallCap) overflow = true;
						__syncwarp();
					}
				}
				fs = next;
				fe = count;
			}
		}
		__syncwarp();
		int* out = members + (size_t)(i - first) * cap;
		if (overflow) {
			if (lane == 0) counts[i - first] = -1;   // built on the host
		}
		else if (count <= cap) {
			for (int t = lane; t < count; t += 32) out[t] = col[t];
			if (lane == 0) counts[i - first] = count;
		}
		else {
			// farthest point: start at the candidate farthest from the leader; each pick
			// lowers the others' distance-to-picked; next = first maximum; taken = -1
			const float* ci = rest3 + 3 * (size_t)i;
			float bv = -1.0f;
			int bm = -1;
			for (int t = lane; t < count; t += 32) {
				const float dd = build_dist2(rest3 + 3 * (size_t)col[t], ci);
				md[t] = dd;
				if (dd > bv) { bv = dd; bm = t; }
			}
			build_argmax(bv, bm);
			int cur = bm, picks = 0;
			for (int t = 0; t < cap; ++t) {
				__syncwarp();
				if (lane == 0) { out[t] = col[cur]; md[cur] = -1.0f; }
				++picks;
				__syncwarp();
				const float* cp = rest3 + 3 * (size_t)col[cur];
				float nv = -1.0f;
				int nm = -1;
				for (int u = lane; u < count; u += 32) {
					float v = md[u];
					if (v < 0.0f) continue;
					const float dd = build_dist2(rest3 + 3 * (size_t)col[u], cp);
					if (dd < v) { v = dd; md[u] = dd; }
					if (v > nv) { nv = v; nm = u; }
				}
				build_argmax(nv, nm);
				if (nm < 0) break;
				cur = nm;
			}
			if (lane == 0) counts[i - first] = picks;
		}
		__syncwarp();
	}
}

// ===========================================================================
// Object mode: rigid shape keeping per object (graph component of at least 50
// Gaussians), once per step right after predict (forward.cu:12141-12166, the device path
// 6829-6958 and 11671-11702).  The per-object sums are in FP64 like the reference's; they
// are reduced in a fixed order (block partials, then one block per object) instead of
// with atomics, so a run repeats bit for bit.
// ===========================================================================
constexpr int kObjMaxK = 64;   // objects with the device path (OBJ_GPU_MAX_K, forward.cu:192)

// objectShapeAccumKernel (forward.cu:6829-6885): per Gaussian of an object, d = p - s
// (s: the object's previous centroid) and d q^T (q = rest - rest centroid); with
// attachment weights (stride 16) every term times w, plus w and w q.  Writes the block's
// sums of objects k0 .. k0 + kc - 1 (kc <= 64) to partial[block][object][stride].
__global__ void __launch_bounds__(kBlock) k_obj_accum(int n, const float4* __restrict__ pos,
	const int* __restrict__ obj_id, const double* __restrict__ q3, const double* __restrict__ shift, int K, int k0,
	int kc, const float* __restrict__ weight, int stride, double* __restrict__ partial)
{
	__shared__ double sh[kObjMaxK * 16];
	for (int t = threadIdx.x; t < kc * stride; t += blockDim.x) sh[t] = 0.0;
	__syncthreads();
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	const int gid = (idx < n) ? obj_id[idx] : -1;
	const int id = (gid >= k0 && gid < k0 + kc) ? gid - k0 : -1;   // index within this chunk
	double v[16];
#pragma unroll
	for (int k = 0; k < 16; ++k) v[k] = 0.0;
	if (id >= 0) {
		const float4 p = pos[idx];
		const double dx = (double)p.x - shift[3 * gid], dy = (double)p.y - shift[3 * gid + 1],
			dz = (double)p.z - shift[3 * gid + 2];
		const double qx = q3[3 * (size_t)idx], qy = q3[3 * (size_t)idx + 1], qz = q3[3 * (size_t)idx + 2];
		v[0] = dx; v[1] = dy; v[2] = dz;
		v[3] = dx * qx; v[4] = dx * qy; v[5] = dx * qz;
		v[6] = dy * qx; v[7] = dy * qy; v[8] = dy * qz;
		v[9] = dz * qx; v[10] = dz * qy; v[11] = dz * qz;
		if (weight) {
			const double w = (double)weight[idx];
#pragma unroll
			for (int k = 0; k < 12; ++k) v[k] *= w;
			v[12] = w; v[13] = w * qx; v[14] = w * qy; v[15] = w * qz;
		}
	}
	const unsigned int full = 0xffffffffu;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int id0 = __shfl_sync(full, id, 0);
	const bool uniform = __all_sync(full, id == id0);
	if (uniform && id0 >= 0) {
		for (int k = 0; k < stride; ++k)
			for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(full, v[k], o);
	}
	// warps add their sums one after another (fixed order); a warp spanning objects adds
	// lane by lane
	for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
		if (warp == w) {
			if (uniform) {
				if (lane == 0 && id0 >= 0)
					for (int k = 0; k < stride; ++k) sh[id0 * stride + k] += v[k];
			}
			else {
				for (int l = 0; l < 32; ++l) {
					const int idl = __shfl_sync(full, id, l);
					for (int k = 0; k < stride; ++k) {
						const double vl = __shfl_sync(full, v[k], l);
						if (lane == 0 && idl >= 0) sh[idl * stride + k] += vl;
					}
				}
			}
		}
		__syncthreads();
	}
	for (int t = threadIdx.x; t < kc * stride; t += blockDim.x)
		partial[((size_t)blockIdx.x * K + k0) * stride + t] = sh[t];
}

// objectShapeSolveKernel (forward.cu:6887-6958), one block per object: the block sums
// the partials in order, then one thread forms c = s + sum d / W, A = sum d q^T - (c - s)
// (sum q)^T, normalises it (Frobenius), takes its rotation with the FP64 polar
// decomposition of shape matching, and writes params = (rest centroid, c, R row-major,
// valid); s becomes c and disp the centroid's move.
__global__ void __launch_bounds__(256) k_obj_solve(int blocks, int K, const double* __restrict__ partial, int stride,
	const int* __restrict__ count, const double* __restrict__ sumq, const float* __restrict__ c0,
	double* __restrict__ shift, float* __restrict__ params, float* __restrict__ disp)
{
	const int k = blockIdx.x;
	__shared__ double red[256];
	__shared__ double S[16];
	for (int c = 0; c < stride; ++c) {
		double acc = 0.0;
		for (int b = threadIdx.x; b < blocks; b += blockDim.x) acc += partial[((size_t)b * K + k) * stride + c];
		red[threadIdx.x] = acc;
		__syncthreads();
		for (int o = blockDim.x / 2; o > 0; o >>= 1) {
			if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
			__syncthreads();
		}
		if (threadIdx.x == 0) S[c] = red[0];
		__syncthreads();
	}
	if (threadIdx.x != 0) return;
	float* Pk = params + 16 * k;
	const int n = count[k];
	if (n < 4) { Pk[15] = 0.0f; disp[k] = 0.0f; return; }
	const bool wOn = (stride == 16);
	const double W = wOn ? S[12] : (double)n;
	if (!(W > 0.0)) { Pk[15] = 0.0f; disp[k] = 0.0f; return; }
	const double inv = 1.0 / W;
	const double dc[3] = { S[0] * inv, S[1] * inv, S[2] * inv };
	const double* sq = wOn ? &S[13] : &sumq[3 * k];
	double a[9];
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c) a[3 * r + c] = S[3 + 3 * r + c] - dc[r] * sq[c];
	double now[3];
	for (int t = 0; t < 3; ++t) {
		now[t] = shift[3 * k + t] + dc[t];
		shift[3 * k + t] = now[t];
	}
	disp[k] = (float)sqrt(dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2]);
	double fn = 0.0;
	for (int t = 0; t < 9; ++t) fn += a[t] * a[t];
	fn = sqrt(fn);
	if (!(fn > 1e-300) || !isfinite(fn)) { Pk[15] = 0.0f; return; }
	M3 A;
	for (int r = 0; r < 3; ++r)
		for (int c = 0; c < 3; ++c) A.m[c][r] = (float)(a[3 * r + c] / fn);
	M3 R;
	if (!shape_rotation_double(A, R)) { Pk[15] = 0.0f; return; }
	for (int t = 0; t < 3; ++t) {
		Pk[t] = wOn ? (float)((double)c0[3 * k + t] + S[13 + t] * inv) : c0[3 * k + t];
		Pk[3 + t] = (float)now[t];
		for (int cc = 0; cc < 3; ++cc) Pk[6 + 3 * t + cc] = R.m[cc][t];
	}
	Pk[15] = 1.0f;
}

// objectShapeMatchKernel (forward.cu:6801-6827): p += s (c + R (x_rest - c0) - p) for the
// free Gaussians of valid objects
__global__ void __launch_bounds__(kBlock) k_obj_match(int n, float4* __restrict__ pos, const float4* __restrict__ rest,
	const int* __restrict__ obj_id, const float* __restrict__ params, float s)
{
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx >= n) return;
	const int id = obj_id[idx];
	const float4 p = pos[idx];
	if (id < 0 || p.w <= 0.0f) return;
	const float* Pk = params + 16 * id;
	if (Pk[15] == 0.0f) return;
	const float4 r = rest[idx];
	const float qx = r.x - Pk[0], qy = r.y - Pk[1], qz = r.z - Pk[2];
	const float gx = Pk[3] + Pk[6] * qx + Pk[7] * qy + Pk[8] * qz;
	const float gy = Pk[4] + Pk[9] * qx + Pk[10] * qy + Pk[11] * qz;
	const float gz = Pk[5] + Pk[12] * qx + Pk[13] * qy + Pk[14] * qz;
	pos[idx] = make_float4(p.x + s * (gx - p.x), p.y + s * (gy - p.y), p.z + s * (gz - p.z), p.w);
}

// object bounding boxes of the predicted positions (objectBoxesKernel, forward.cu:6960-6981):
// float min / max through integer atomics on the bits, block-local first
__device__ __forceinline__ void obj_atomic_min(float* a, float v)
{
	v += 0.0f;
	if (v >= 0.0f) atomicMin((int*)a, __float_as_int(v));
	else atomicMax((unsigned int*)a, __float_as_uint(v));
}
__device__ __forceinline__ void obj_atomic_max(float* a, float v)
{
	v += 0.0f;
	if (v >= 0.0f) atomicMax((int*)a, __float_as_int(v));
	else atomicMin((unsigned int*)a, __float_as_uint(v));
}

__global__ void k_obj_boxes_init(int K, float* __restrict__ boxes)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t < 6 * K) boxes[t] = ((t % 6) < 3) ? FLT_MAX : -FLT_MAX;
}

__global__ void __launch_bounds__(kBlock) k_obj_boxes(int n, const float4* __restrict__ pos,
	const int* __restrict__ obj_id, int K, float* __restrict__ boxes)
{
	__shared__ float sh[kObjMaxK * 6];
	for (int t = threadIdx.x; t < K * 6; t += blockDim.x) sh[t] = ((t % 6) < 3) ? FLT_MAX : -FLT_MAX;
	__syncthreads();
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	if (idx < n) {
		const int id = obj_id[idx];
		const float4 p = pos[idx];
		if (id >= 0 && isfinite(p.x) && isfinite(p.y) && isfinite(p.z)) {
			float* b = &sh[6 * id];
			obj_atomic_min(&b[0], p.x); obj_atomic_min(&b[1], p.y); obj_atomic_min(&b[2], p.z);
			obj_atomic_max(&b[3], p.x); obj_atomic_max(&b[4], p.y); obj_atomic_max(&b[5], p.z);
		}
	}
	__syncthreads();
	for (int t = threadIdx.x; t < K * 6; t += blockDim.x) {
		const float v = sh[t];
		if (v == FLT_MAX || v == -FLT_MAX) continue;
		if ((t % 6) < 3) obj_atomic_min(&boxes[t], v);
		else obj_atomic_max(&boxes[t], v);
	}
}

// selfColActiveKernel (forward.cu:6998-7029): with same-object contacts off, only Gaussians
// whose start or predicted position lies in another object's box (grown by search + 2 x
// the largest centroid move + 2 dc) enter the hash grid; Gaussians of no object always do
__global__ void __launch_bounds__(kBlock) k_sc_active(int n, const StepParams* __restrict__ P,
	const float4* __restrict__ x, const float4* __restrict__ p, const int* __restrict__ obj_id,
	const float* __restrict__ boxes, const float* __restrict__ disp, int K, unsigned char* __restrict__ active,
	DevCounters* __restrict__ ctr)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	float md = 0.0f;
	for (int k = 0; k < K; ++k) md = fmaxf(md, disp[k]);
	const float inflate = P->sc_search + 2.0f * md + 2.0f * P->sc_dc;
	const int id = obj_id[i];
	unsigned char a = 0;
	if (id < 0) {
		a = 1;
	}
	else {
		const float4 pp = p[i], xx = x[i];
		for (int k = 0; k < K; ++k) {
			if (k == id) continue;
			const float* b = &boxes[6 * k];
			const float lx = b[0] - inflate, ly = b[1] - inflate, lz = b[2] - inflate;
			const float hx = b[3] + inflate, hy = b[4] + inflate, hz = b[5] + inflate;
			const bool inP = pp.x >= lx && pp.x <= hx && pp.y >= ly && pp.y <= hy && pp.z >= lz && pp.z <= hz;
			const bool inX = xx.x >= lx && xx.x <= hx && xx.y >= ly && xx.y <= hy && xx.z >= lz && xx.z <= hz;
			if (inP || inX) { a = 1; break; }
		}
	}
	active[i] = a;
	const unsigned int m = __ballot_sync(__activemask(), a != 0);
	if (m && (threadIdx.x & 31) == __ffs(__activemask()) - 1) atomicAdd(&ctr->sc_active, __popc(m));
}

// Contact push (objectContactPush, forward.cu:11858-11890; kernels 7326-7354): per object,
// the mean of the frame's cross-object corrections over the Gaussians that received one,
// times the shape stiffness, is added to the object's other free Gaussians.  Block
// partials of (sum, count) in a fixed order, then one thread per object.
__global__ void __launch_bounds__(kBlock) k_obj_push_sum(int n, const int* __restrict__ obj_id,
	const float4* __restrict__ accum, int K, int k0, int kc, const DevCounters* __restrict__ ctr,
	float* __restrict__ partial)
{
	__shared__ float sh[kObjMaxK * 4];
	if (ctr->sc_contacts == 0u) return;
	for (int t = threadIdx.x; t < kc * 4; t += blockDim.x) sh[t] = 0.0f;
	__syncthreads();
	const int idx = blockIdx.x * blockDim.x + threadIdx.x;
	int id = -1;
	float4 a = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
	if (idx < n) {
		const int gid = obj_id[idx];
		id = (gid >= k0 && gid < k0 + kc) ? gid - k0 : -1;
		a = accum[idx];
		if (!(a.x * a.x + a.y * a.y + a.z * a.z > 1e-30f)) id = -1;
	}
	const unsigned int full = 0xffffffffu;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
		if (warp == w) {
			for (int l = 0; l < 32; ++l) {
				const int idl = __shfl_sync(full, id, l);
				const float ax = __shfl_sync(full, a.x, l), ay = __shfl_sync(full, a.y, l), az = __shfl_sync(full, a.z, l);
				if (lane == 0 && idl >= 0) {
					float* S = &sh[4 * idl];
					S[0] += ax; S[1] += ay; S[2] += az; S[3] += 1.0f;
				}
			}
		}
		__syncthreads();
	}
	for (int t = threadIdx.x; t < kc * 4; t += blockDim.x) partial[((size_t)blockIdx.x * K + k0) * 4 + t] = sh[t];
}

__global__ void k_obj_push_solve(int blocks, int K, const float* __restrict__ partial, const DevCounters* __restrict__ ctr,
	float s, float* __restrict__ T)
{
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= K) return;
	T[4 * k + 3] = 0.0f;
	if (ctr->sc_contacts == 0u) return;
	float sum[4] = { 0.0f, 0.0f, 0.0f, 0.0f };
	for (int b = 0; b < blocks; ++b)
		for (int c = 0; c < 4; ++c) sum[c] += partial[((size_t)b * K + k) * 4 + c];
	const float cnt = sum[3];
	if (!(cnt > 0.0f)) return;
	const float sc = s / cnt;
	const float tx = sum[0] * sc, ty = sum[1] * sc, tz = sum[2] * sc;
	if (!isfinite(tx) || !isfinite(ty) || !isfinite(tz)) return;
	T[4 * k] = tx; T[4 * k + 1] = ty; T[4 * k + 2] = tz; T[4 * k + 3] = 1.0f;
}

// objectPushApplyKernel (forward.cu:7341-7354), then the ground plane again
// (groundProjectKernel, forward.cu:7405-7421) when it is on
__global__ void __launch_bounds__(kBlock) k_obj_push_apply(int n, const StepParams* __restrict__ P,
	const int* __restrict__ obj_id, const float4* __restrict__ accum, const float* __restrict__ T,
	const DevCounters* __restrict__ ctr, float4* __restrict__ pos, const float* __restrict__ crg)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	if (ctr->sc_contacts == 0u) return;
	float4 p = pos[i];
	if (p.w <= 0.0f) return;
	bool moved = false;
	const int id = obj_id[i];
	if (id >= 0 && T[4 * id + 3] != 0.0f) {
		const float4 a = accum[i];
		if (!(a.x * a.x + a.y * a.y + a.z * a.z > 1e-30f)) {
			p.x = p.x + T[4 * id]; p.y = p.y + T[4 * id + 1]; p.z = p.z + T[4 * id + 2];
			moved = true;
		}
	}
	if (P->ground_on) {
		const float c = P->gn[0] * p.x + P->gn[1] * p.y + P->gn[2] * p.z - P->ground_plane - (crg ? crg[i] : 0.0f);
		if (c < 0.0f) {
			p.x = p.x - c * P->gn[0]; p.y = p.y - c * P->gn[1]; p.z = p.z - c * P->gn[2];
			moved = true;
		}
	}
	if (moved) pos[i] = p;
}

// ===========================================================================
// ChainMail displacement propagation (runChainmailGPU's dense path,
// forward.cu:12808-13006): arrival-time sweeps that move each Gaussian toward the
// neighbour that reached it first, then relax sweeps.
//
// Layout: td[i] = (arrival time, density) as one float2, so a neighbour costs one
// 8-byte load; positions are the engine's float4 (inverse mass in w, untouched).
//
// Propagation runs as a frontier sweep.  A Gaussian can change in a sweep only if a
// neighbour's arrival time dropped in the sweep before (otherwise its time is already
// no later than every neighbour's offer, so the reference kernel writes its input back
// unchanged), so each sweep visits only the neighbours of the Gaussians flagged in the
// previous one: k_cm_expand turns the flags into a work list (warp ballots give one
// atomic per warp), k_cm_sweep computes the reference kernel's output for the listed
// Gaussians from the unchanged state, k_cm_commit writes back the ones that improved
// and flags them for the next sweep.  The result equals the reference's dense Jacobi
// sweep exactly; when a quarter of the Gaussians are flagged the list is replaced by
// all Gaussians.
// ===========================================================================
constexpr float kCmAir = 0.13f, kCmSkin = 0.45f, kCmBone = 0.75f;   // forward.h:63-65

struct CmMaterial {                 // setChainmailMaterialParams (forward.cu:4844-4858)
	float global, air, skin, bone, influence;
	int use_edge;
};

struct CmState {                    // device-side sweep bookkeeping
	int pending;                    // Gaussians flagged by the last sweep or by seeds
	int work;                       // entries in the work list of this sweep
	int dense;                      // this sweep visits every Gaussian
	int pad;
};

// cm_getConstraint (forward.cu:5221-5264): axis tolerance of a density class
__device__ __forceinline__ float cm_axis_tol(const CmMaterial& M, float density)
{
	const float c = (density < kCmAir) ? M.air : ((density < kCmSkin) ? M.skin : M.bone);
	return c * fmaxf(1e-4f, M.global);
}

// cm_edgeScaleFromStiff (forward.cu:5266-5278)
__device__ __forceinline__ float cm_edge_scale(const CmMaterial& M, float stiff)
{
	if (!M.use_edge || M.influence <= 0.0f) return 1.0f;
	const float s = fminf(fmaxf(stiff, 0.05f), 1.0f);
	const float t = (s - 0.05f) / 0.95f;
	const float scale = 1.0f + M.influence * (t * 2.0f - 1.0f);
	return fminf(fmaxf(scale, 0.1f), 4.0f);
}

__device__ __forceinline__ float cm_class_time(float d)
{
	return (d < kCmAir) ? 1.0f : ((d < kCmSkin) ? 0.3f : ((d < kCmBone) ? 0.05f : 0.005f));
}

// cm_propagationTime (forward.cu:5280-5293)
__device__ __forceinline__ float cm_link_time(float d0, float d1)
{
	return (cm_class_time(d0) + cm_class_time(d1)) * 0.5f;
}

// cm_correctionFromNeighbor (forward.cu:5295-5330)
__device__ __forceinline__ float3 cm_correction(const CmMaterial& M, float3 epos, float3 npos, float targ, float ndens,
	float stiff)
{
	const float dx = cm_axis_tol(M, ndens);
	const float edge_scale = cm_edge_scale(M, stiff);
	const float3 dir = sub3(epos, npos);
	const float len = len3(dir);
	if (len < 1e-6f) return make_float3(0.0f, 0.0f, 0.0f);
	const float inv_len = 1.0f / len;
	const float3 nd = mul3(dir, inv_len);
	if (len < targ - dx) return mul3(nd, ((targ - dx) - len) * edge_scale);
	if (len > targ + dx) return mul3(nd, -((len - (targ + dx)) * edge_scale));
	return make_float3(0.0f, 0.0f, 0.0f);
}

// seeds, in order (applySeedCommandsKernel, forward.cu:5907-5924): move by delta, arrival
// time 0, flagged for the next sweep
__global__ void k_cm_seed(int count, const int* __restrict__ idx, const float* __restrict__ delta,
	float4* __restrict__ pos, float2* __restrict__ td, unsigned char* __restrict__ flag, CmState* __restrict__ st)
{
	if (blockIdx.x != 0 || threadIdx.x != 0) return;
	for (int k = 0; k < count; ++k) {
		const int i = idx[k];
		float4 p = pos[i];
		p.x = p.x + delta[3 * k]; p.y = p.y + delta[3 * k + 1]; p.z = p.z + delta[3 * k + 2];
		pos[i] = p;
		td[i].x = 0.0f;
		if (!flag[i]) { flag[i] = 1; ++st->pending; }
	}
}

// start of a sweep: dense when more than `dense_above` Gaussians are flagged
__global__ void k_cm_begin(int n, int dense_above, CmState* __restrict__ st)
{
	const int dense = st->pending > dense_above;
	st->dense = dense;
	st->work = dense ? n : 0;
	st->pending = 0;
}

// Work list of this sweep: the neighbours of every flagged Gaussian, each once (a bit
// per Gaussian in `mark`), appended with one atomic per warp; clears the flags.  The
// lanes of a warp walk the rows of the warp's flagged Gaussians together.
__global__ void __launch_bounds__(kBlock) k_cm_expand(int n, const int* __restrict__ off, const int* __restrict__ nbr,
	unsigned char* __restrict__ flag, unsigned int* __restrict__ mark, int* __restrict__ work, CmState* __restrict__ st)
{
	const bool dense = st->dense != 0;
	const int lane = threadIdx.x & 31;
	const int stride = gridDim.x * blockDim.x;
	for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
		const int i = base + lane;
		const bool pending = i < n && flag[i];
		if (pending) flag[i] = 0;
		if (dense) continue;
		unsigned int todo = __ballot_sync(0xffffffffu, pending);
		while (todo) {
			const int p = base + __ffs(todo) - 1;
			todo &= todo - 1;
			const int e1 = off[p + 1];
			for (int e0 = off[p]; e0 < e1; e0 += 32) {
				const int e = e0 + lane;
				bool fresh = false;
				int j = 0;
				if (e < e1) {
					j = __ldg(nbr + e);
					if (j >= 0 && j < n) {
						const unsigned int bit = 1u << (j & 31);
						fresh = (atomicOr(mark + (j >> 5), bit) & bit) == 0u;
					}
				}
				const unsigned int fm = __ballot_sync(0xffffffffu, fresh);
				if (fm) {
					int at = 0;
					if (lane == 0) at = atomicAdd(&st->work, __popc(fm));
					at = __shfl_sync(0xffffffffu, at, 0);
					if (fresh) work[at + __popc(fm & ((1u << lane) - 1u))] = j;
				}
			}
		}
	}
}

// chainmailPropagateKernelBest (forward.cu:5396-5464) for the listed Gaussians: the
// earliest arrival through any neighbour; when it beats the Gaussian's own time, one
// correction toward the neighbour it came through.  Reads the state only; results go
// to per-entry scratch (Jacobi: every entry sees the state before this sweep).
__global__ void __launch_bounds__(kBlock) k_cm_sweep(int n, const float4* __restrict__ pos,
	const float2* __restrict__ td, const int* __restrict__ off, const int* __restrict__ nbr,
	const float* __restrict__ ndist, const float* __restrict__ nstiff, const int* __restrict__ work,
	const CmState* __restrict__ st, CmMaterial M, float strength, float4* __restrict__ out_pos,
	float* __restrict__ out_time)
{
	const int cnt = st->work;
	const bool dense = st->dense != 0;
	const int stride = gridDim.x * blockDim.x;
	for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += stride) {
		const int i = dense ? k : work[k];
		const float4 e4 = ld4(pos, i);
		const float2 me = td[i];
		const float edens = me.y, tcur = me.x;
		float best_time = tcur, best_dist = 0.0f, best_dens = 0.0f;
		int best = -1;
		const int e0 = off[i], e1 = off[i + 1];
		for (int e = e0; e < e1; ++e) {
			const int j = __ldg(nbr + e);
			const float2 o = td[j];
			const float cand = o.x + cm_link_time(edens, o.y);
			if (cand < best_time) { best_time = cand; best = j; best_dist = __ldg(ndist + e); best_dens = o.y; }
		}
		float4 out = e4;
		if (best >= 0 && best_time < tcur) {
			float stiff = 1.0f;
			for (int e = e0; e < e1; ++e)
				if (__ldg(nbr + e) == best) { stiff = __ldg(nstiff + e); break; }
			const float3 epos = f3(e4);
			const float3 corr = cm_correction(M, epos, f3(ld4(pos, best)), best_dist, best_dens, stiff);
			if (len3(corr) > 0.0f) {
				const float3 o = add3(epos, mul3(corr, strength));
				out = make_float4(o.x, o.y, o.z, e4.w);
			}
		}
		out_pos[k] = out;
		out_time[k] = best_time;
	}
}

// Writes back the entries whose arrival time dropped, flags them for the next sweep and
// clears the work-list marks.
__global__ void __launch_bounds__(kBlock) k_cm_commit(int n, float4* __restrict__ pos, float2* __restrict__ td,
	const int* __restrict__ work, const float4* __restrict__ out_pos, const float* __restrict__ out_time,
	unsigned char* __restrict__ flag, unsigned int* __restrict__ mark, CmState* __restrict__ st)
{
	const int cnt = st->work;
	const bool dense = st->dense != 0;
	const int lane = threadIdx.x & 31;
	const int stride = gridDim.x * blockDim.x;
	for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < cnt; base += stride) {
		const int k = base + lane;
		bool improved = false;
		if (k < cnt) {
			const int i = dense ? k : work[k];
			if (!dense) atomicAnd(mark + (i >> 5), ~(1u << (i & 31)));
			const float t = out_time[k];
			if (t < td[i].x) {
				pos[i] = out_pos[k];
				td[i].x = t;
				flag[i] = 1;
				improved = true;
			}
		}
		const unsigned int fm = __ballot_sync(0xffffffffu, improved);
		if (fm && lane == 0) atomicAdd(&st->pending, __popc(fm));
	}
}

// chainmailRelaxKernel (forward.cu:5466-5559): every Gaussian toward the rest lengths of
// its edges, mean correction clamped to 1.5 x the mean rest length, stiffness, damping.
__global__ void __launch_bounds__(kBlock) k_cm_relax(int n, const float4* __restrict__ pin, float4* __restrict__ pout,
	const float2* __restrict__ td, const int* __restrict__ off, const int* __restrict__ nbr,
	const float* __restrict__ ndist, const float* __restrict__ nstiff, CmMaterial M, float stiffness, float damping)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float4 e4 = ld4(pin, i);
	const float3 epos = f3(e4);
	const float etol = cm_axis_tol(M, td[i].y);
	float3 acc = make_float3(0.0f, 0.0f, 0.0f);
	int corr_count = 0, dist_count = 0;
	float sum_target = 0.0f;
	const int e0 = off[i], e1 = off[i + 1];
	for (int e = e0; e < e1; ++e) {
		const int j = __ldg(nbr + e);
		const float3 npos = f3(ld4(pin, j));
		const float ntol = cm_axis_tol(M, td[j].y);
		const float edge_scale = cm_edge_scale(M, __ldg(nstiff + e));
		const float targ = __ldg(ndist + e);
		const float tol = (0.0000001f * (etol + ntol)) / edge_scale;
		const float3 dir = sub3(npos, epos);
		const float len = len3(dir);
		if (len < 1e-6f) continue;
		const float inv_len = 1.0f / len;
		const float3 nd = mul3(dir, inv_len);
		if (len < targ - tol) {
			acc = sub3(acc, mul3(nd, ((targ - tol) - len) * edge_scale));
			corr_count++;
		}
		else if (len > targ + tol) {
			acc = add3(acc, mul3(nd, (len - (targ + tol)) * edge_scale));
			corr_count++;
		}
		sum_target += targ;
		dist_count++;
	}
	if (corr_count > 0) {
		float3 avg = mul3(acc, 1.0f / (float)corr_count);
		float max_step = 0.6f;
		if (dist_count > 0) max_step = 1.5f * (sum_target / (float)dist_count);
		const float cl = len3(avg);
		if (cl > 1e-6f && cl > max_step) avg = mul3(avg, max_step / cl);
		const float3 corrected = add3(epos, mul3(avg, stiffness));
		const float3 o = add3(epos, mul3(sub3(corrected, epos), 1.0f - damping));
		pout[i] = make_float4(o.x, o.y, o.z, e4.w);
	}
	else {
		pout[i] = e4;
	}
}

// arrival times (caller order) and the caller-order position mirror after a run
__global__ void __launch_bounds__(kBlock) k_cm_publish(int n, const float4* __restrict__ pos,
	const float2* __restrict__ td, const int* __restrict__ perm, float* __restrict__ pos_out3,
	float* __restrict__ time_out)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const int o = perm ? perm[i] : i;
	const float4 p = pos[i];
	if (pos_out3) { pos_out3[3 * (size_t)o] = p.x; pos_out3[3 * (size_t)o + 1] = p.y; pos_out3[3 * (size_t)o + 2] = p.z; }
	if (time_out) time_out[o] = td[i].x;
}

}  // namespace dev
}  // namespace xpbd
