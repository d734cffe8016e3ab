// Headless 3DGS splatting of the solver's Gaussians into a device image: the
// published tile rasteriser (Kerbl et al. 2023) behind the reference viewer
// (preprocessCUDA / renderCUDA, forward.cu:1919-2650; binning in
// rasterizer_impl.cu:53-140, 201-470), forward pass only.
//
//   prepare  one thread per Gaussian: near-plane and box culling, projection to pixels,
//            3D covariance R S S^T R^T, EWA 2D covariance J W Sigma W^T J^T + 0.3 px,
//            conic, 3-sigma radius, touched 16x16 tiles, colour (spherical harmonics
//            toward the camera, or given RGB)
//   order    Gaussians sorted by view depth (stable), then (tile, Gaussian) pairs
//            written in depth order and stable-sorted by tile alone: the same order as
//            the reference's stable sort of (tile << 32 | depth) pairs generated in
//            Gaussian order, with a 10-14 bit tile key instead of a 45-bit one
//   tiles    one 256-thread block per tile, Gaussians staged 256 at a time in shared
//            memory, front-to-back alpha compositing with early termination; image
//            channel-major (3 x H x W) plus transmittance, contributor count, the
//            first Gaussian with alpha > 0.1 (picking) and an optional checker floor
//            in place of the background (renderCUDA's ground composite)
//
// Camera matrices are column-major 4x4 (world -> view, world -> clip), view space looks
// down +z, pixel centres at integer coordinates.
#pragma once
#include "kernels.cuh"

namespace xpbd {
namespace dev {

constexpr int kTile = 16;
constexpr int kTilePix = kTile * kTile;

struct RenderFrame {
	float view[16], proj[16];
	float campos[3];
	float tan_fovx, tan_fovy, focal_x, focal_y;
	float scale_mod;
	float box_lo[3], box_hi[3];
	float bg[3];
	int W, H, tiles_x, tiles_y;
	int sh_deg;        // -1: colours are RGB per Gaussian; 0..3: SH degree
	int sh_coeffs;     // coefficients (RGB triples) per Gaussian in the colour array
	int antialias;
	int pick;
	// checker floor (renderCUDA's ground composite; floor_on = 0 keeps the background)
	int floor_on;
	float fl_cam[3], fl_rx[3], fl_ry[3], fl_rz[3], fl_n[3], fl_t1[3], fl_t2[3], fl_origin[3];
	float fl_camh, fl_pix, fl_inv_fade2;
};

// real spherical harmonics of degree <= 3 (the basis of the 3DGS colour model):
// c0 = 1/(2 sqrt(pi)), c1 = sqrt(3/(4 pi)), c2 and c3 the normalisations of the
// l = 2 and l = 3 real harmonics in Cartesian form
__device__ __forceinline__ float3 sh_color(int deg, const float* __restrict__ c, float3 d)
{
	const float c0 = 0.28209479177387814f, c1 = 0.4886025119029199f;
	float r = c0 * c[0], g = c0 * c[1], b = c0 * c[2];
	if (deg > 0) {
		const float x = d.x, y = d.y, z = d.z;
		r = r - c1 * y * c[3] + c1 * z * c[6] - c1 * x * c[9];
		g = g - c1 * y * c[4] + c1 * z * c[7] - c1 * x * c[10];
		b = b - c1 * y * c[5] + c1 * z * c[8] - c1 * x * c[11];
		if (deg > 1) {
			const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
			const float w2[5] = { 1.0925484305920792f * xy, -1.0925484305920792f * yz,
				0.31539156525252005f * (2.0f * zz - xx - yy), -1.0925484305920792f * xz,
				0.5462742152960396f * (xx - yy) };
			for (int k = 0; k < 5; ++k) {
				r += w2[k] * c[3 * (4 + k)];
				g += w2[k] * c[3 * (4 + k) + 1];
				b += w2[k] * c[3 * (4 + k) + 2];
			}
			if (deg > 2) {
				const float w3[7] = { -0.5900435899266435f * y * (3.0f * xx - yy), 2.890611442640554f * xy * z,
					-0.4570457994644658f * y * (4.0f * zz - xx - yy),
					0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy),
					-0.4570457994644658f * x * (4.0f * zz - xx - yy), 1.445305721320277f * z * (xx - yy),
					-0.5900435899266435f * x * (xx - 3.0f * yy) };
				for (int k = 0; k < 7; ++k) {
					r += w3[k] * c[3 * (9 + k)];
					g += w3[k] * c[3 * (9 + k) + 1];
					b += w3[k] * c[3 * (9 + k) + 2];
				}
			}
		}
	}
	return make_float3(fmaxf(r + 0.5f, 0.0f), fmaxf(g + 0.5f, 0.0f), fmaxf(b + 0.5f, 0.0f));
}

// Per Gaussian: pixel centre, conic + opacity, colour, depth sort key (0xffffffff when
// culled), radius and tile rectangle.  Quaternions are (w, x, y, z), used as given.
__global__ void __launch_bounds__(kBlock) k_splat_prepare(int n, RenderFrame F, const float* __restrict__ pos,
	const float* __restrict__ scales, const float* __restrict__ quats, const float* __restrict__ opacity,
	const float* __restrict__ colors, float4* __restrict__ xy, float4* __restrict__ conic_op,
	float4* __restrict__ rgb, unsigned int* __restrict__ dkey, int* __restrict__ radii, int4* __restrict__ rect,
	int* __restrict__ touched)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	radii[i] = 0;
	touched[i] = 0;
	dkey[i] = 0xffffffffu;
	const float3 p = make_float3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
	const float* V = F.view;
	const float vx = V[0] * p.x + V[4] * p.y + V[8] * p.z + V[12];
	const float vy = V[1] * p.x + V[5] * p.y + V[9] * p.z + V[13];
	const float vz = V[2] * p.x + V[6] * p.y + V[10] * p.z + V[14];
	if (vz <= 0.2f) return;
	if (p.x < F.box_lo[0] || p.y < F.box_lo[1] || p.z < F.box_lo[2] || p.x > F.box_hi[0] || p.y > F.box_hi[1] ||
		p.z > F.box_hi[2])
		return;
	const float* P = F.proj;
	const float hx = P[0] * p.x + P[4] * p.y + P[8] * p.z + P[12];
	const float hy = P[1] * p.x + P[5] * p.y + P[9] * p.z + P[13];
	const float hw = P[3] * p.x + P[7] * p.y + P[11] * p.z + P[15];
	const float iw = 1.0f / (hw + 0.0000001f);
	// pixel coordinate of an NDC value, evaluated in double as the reference's ndc2Pix
	const float px = (float)((((double)(hx * iw) + 1.0) * F.W - 1.0) * 0.5);
	const float py = (float)((((double)(hy * iw) + 1.0) * F.H - 1.0) * 0.5);
	// Sigma = R diag(s^2) R^T, R the rotation of the quaternion
	const float qr = quats[4 * i], qx = quats[4 * i + 1], qy = quats[4 * i + 2], qz = quats[4 * i + 3];
	const float R[3][3] = { { 1.f - 2.f * (qy * qy + qz * qz), 2.f * (qx * qy - qr * qz), 2.f * (qx * qz + qr * qy) },
		{ 2.f * (qx * qy + qr * qz), 1.f - 2.f * (qx * qx + qz * qz), 2.f * (qy * qz - qr * qx) },
		{ 2.f * (qx * qz - qr * qy), 2.f * (qy * qz + qr * qx), 1.f - 2.f * (qx * qx + qy * qy) } };
	const float s0 = F.scale_mod * scales[3 * i], s1 = F.scale_mod * scales[3 * i + 1],
				s2 = F.scale_mod * scales[3 * i + 2];
	float M[3][3];   // M = diag(s) R^T, Sigma = M^T M
	for (int c = 0; c < 3; ++c) {
		M[0][c] = s0 * R[c][0];
		M[1][c] = s1 * R[c][1];
		M[2][c] = s2 * R[c][2];
	}
	float S[6];      // xx xy xz yy yz zz
	{
		int k = 0;
		for (int a = 0; a < 3; ++a)
			for (int b = a; b < 3; ++b) S[k++] = M[0][a] * M[0][b] + M[1][a] * M[1][b] + M[2][a] * M[2][b];
	}
	// EWA: cov2 = T Sigma T^T, T = J W (perspective Jacobian at the clamped view point,
	// W the view rotation)
	const float limx = 1.3f * F.tan_fovx, limy = 1.3f * F.tan_fovy;
	const float tx = fminf(limx, fmaxf(-limx, vx / vz)) * vz;
	const float ty = fminf(limy, fmaxf(-limy, vy / vz)) * vz;
	const float j00 = F.focal_x / vz, j02 = -(F.focal_x * tx) / (vz * vz);
	const float j11 = F.focal_y / vz, j12 = -(F.focal_y * ty) / (vz * vz);
	float T0[3], T1[3];
	for (int c = 0; c < 3; ++c) {
		T0[c] = j00 * V[4 * c] + j02 * V[4 * c + 2];
		T1[c] = j11 * V[4 * c + 1] + j12 * V[4 * c + 2];
	}
	const float Sm[3][3] = { { S[0], S[1], S[2] }, { S[1], S[3], S[4] }, { S[2], S[4], S[5] } };
	float u0[3], u1[3];   // Sigma T0, Sigma T1
	for (int a = 0; a < 3; ++a) {
		u0[a] = Sm[a][0] * T0[0] + Sm[a][1] * T0[1] + Sm[a][2] * T0[2];
		u1[a] = Sm[a][0] * T1[0] + Sm[a][1] * T1[1] + Sm[a][2] * T1[2];
	}
	float ca = T0[0] * u0[0] + T0[1] * u0[1] + T0[2] * u0[2];
	const float cb = T0[0] * u1[0] + T0[1] * u1[1] + T0[2] * u1[2];
	float cc = T1[0] * u1[0] + T1[1] * u1[1] + T1[2] * u1[2];
	const float det0 = ca * cc - cb * cb;
	ca += 0.3f;
	cc += 0.3f;
	const float det = ca * cc - cb * cb;
	const float aa = F.antialias ? sqrtf(fmaxf(0.000025f, det0 / det)) : 1.0f;
	if (det == 0.0f) return;
	const float idet = 1.0f / det;
	const float mid = 0.5f * (ca + cc);
	const float l1 = mid + sqrtf(fmaxf(0.1f, mid * mid - det));
	const float l2 = mid - sqrtf(fmaxf(0.1f, mid * mid - det));
	const int radius = (int)ceilf(3.0f * sqrtf(fmaxf(l1, l2)));
	const int x0 = min(F.tiles_x, max(0, (int)((px - radius) / kTile)));
	const int y0 = min(F.tiles_y, max(0, (int)((py - radius) / kTile)));
	const int x1 = min(F.tiles_x, max(0, (int)((px + radius + kTile - 1) / kTile)));
	const int y1 = min(F.tiles_y, max(0, (int)((py + radius + kTile - 1) / kTile)));
	const int cnt = (x1 - x0) * (y1 - y0);
	if (cnt == 0) return;
	float3 col;
	if (F.sh_deg >= 0) {
		float dx = p.x - F.campos[0], dy = p.y - F.campos[1], dz = p.z - F.campos[2];
		const float len = sqrtf(dx * dx + dy * dy + dz * dz);
		dx /= len; dy /= len; dz /= len;
		const float* src = colors + (size_t)3 * F.sh_coeffs * i;
		float c[48];
		if (F.sh_deg == 3 || F.sh_deg == 1) {
			// 192 or 48 bytes per Gaussian: 16-byte aligned rows, read as float4
			const float4* s4 = reinterpret_cast<const float4*>(src);
			const int n4 = F.sh_deg == 3 ? 12 : 3;
#pragma unroll
			for (int k = 0; k < 12; ++k)
				if (k < n4) {
					const float4 v = __ldg(s4 + k);
					c[4 * k] = v.x; c[4 * k + 1] = v.y; c[4 * k + 2] = v.z; c[4 * k + 3] = v.w;
				}
		} else {
#pragma unroll
			for (int k = 0; k < 27; ++k)
				if (k < 3 * F.sh_coeffs) c[k] = __ldg(src + k);
		}
		col = sh_color(F.sh_deg, c, make_float3(dx, dy, dz));
	} else {
		col = make_float3(colors[3 * i], colors[3 * i + 1], colors[3 * i + 2]);
	}
	// half widths of the box outside which alpha stays below 1/255: the ellipse
	// d^T Q d <= 2 ln(255 o) (Q the conic, Q^-1 the low-passed 2D covariance) has the
	// axis-aligned half widths sqrt(t cov_xx), sqrt(t cov_yy); the margins keep the
	// compositing kernel's region test conservative under FP32 rounding
	const float o_eff = opacity[i] * aa;
	float ex = -1.0f, ey = -1.0f;
	if (!(det > 0.0f)) {
		ex = ey = FLT_MAX;
	} else if (o_eff >= 1.0f / 255.0f) {
		const float t = 2.0f * logf(255.0f * o_eff) * 1.002f + 0.02f;
		ex = sqrtf(t * ca) * 1.001f + 0.01f;
		ey = sqrtf(t * cc) * 1.001f + 0.01f;
	}
	xy[i] = make_float4(px, py, ex, ey);
	conic_op[i] = make_float4(cc * idet, -cb * idet, ca * idet, o_eff);
	rgb[i] = make_float4(col.x, col.y, col.z, 0.0f);
	dkey[i] = __float_as_uint(vz);   // positive floats order as unsigned integers
	radii[i] = radius;
	rect[i] = make_int4(x0, y0, x1, y1);
	touched[i] = cnt;
}

// total tiles touched (the pair count), accumulated into *total (zeroed before)
__global__ void __launch_bounds__(kBlock) k_splat_total(int n, const int* __restrict__ touched,
	unsigned long long* __restrict__ total)
{
	__shared__ unsigned long long s_part[kBlock / 32];
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long v = i < n ? (unsigned long long)touched[i] : 0ull;
	for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
	if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = v;
	__syncthreads();
	if (threadIdx.x == 0) {
		unsigned long long t = 0;
		for (int w = 0; w < kBlock / 32; ++w) t += s_part[w];
		if (t) atomicAdd(total, t);
	}
}

__global__ void __launch_bounds__(kBlock) k_iota(int n, int* __restrict__ a)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) a[i] = i;
}

// tiles touched by the Gaussians in depth order (scan input)
__global__ void __launch_bounds__(kBlock) k_splat_counts(int n, const int* __restrict__ order,
	const int* __restrict__ touched, long long* __restrict__ cnt)
{
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k < n) cnt[k] = touched[order[k]];
}

// One (tile, Gaussian) pair per touched tile, Gaussians in depth order, tiles of a
// Gaussian row by row.  A warp takes 32 consecutive Gaussians of the depth order and
// writes their pairs together, lane j the j-th pair of each 32, so that the stores of
// a warp are consecutive; each lane finds the Gaussian owning its pair by a binary
// search over the warp's prefix offsets (shuffles).
template <typename Key>
__global__ void __launch_bounds__(kBlock) k_splat_pairs(int n, const int* __restrict__ order,
	const long long* __restrict__ offs, const int4* __restrict__ rect, int tiles_x, Key* __restrict__ tkey,
	int* __restrict__ val)
{
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	const int lane = threadIdx.x & 31;
	if (k - lane >= n) return;                       // whole warp past the end
	const long long s0 = offs[min(k, n)];
	const long long e0 = k < n ? offs[k + 1] : s0;
	int g = 0;
	int4 r = make_int4(0, 0, 1, 1);
	if (e0 > s0) {
		g = order[k];
		r = rect[g];
	}
	const long long base = __shfl_sync(0xffffffffu, s0, 0);
	const long long total = __shfl_sync(0xffffffffu, e0, 31) - base;
	const int loc = (int)(s0 - base);                // this lane's first pair within the warp's run
	for (long long p0 = 0; p0 < total; p0 += 32) {
		const int p = (int)p0 + lane;
		int owner = 0;                               // largest lane whose run starts at or before p
		for (int step = 16; step > 0; step >>= 1) {
			const int cand = owner + step;
			const int lc = __shfl_sync(0xffffffffu, loc, cand & 31);
			if (cand < 32 && lc <= p) owner = cand;
		}
		const int o_loc = __shfl_sync(0xffffffffu, loc, owner);
		const int o_g = __shfl_sync(0xffffffffu, g, owner);
		const int o_x0 = __shfl_sync(0xffffffffu, r.x, owner);
		const int o_y0 = __shfl_sync(0xffffffffu, r.y, owner);
		const int o_x1 = __shfl_sync(0xffffffffu, r.z, owner);
		if (p < total) {
			const int li = p - o_loc, w = o_x1 - o_x0;
			const int y = o_y0 + li / w, x = o_x0 + li % w;
			tkey[base + p] = (Key)(y * tiles_x + x);
			val[base + p] = o_g;
		}
	}
}

// [start, end) of every tile in the sorted pair list: two lower-bound searches per tile
template <typename Key>
__global__ void __launch_bounds__(kBlock) k_splat_ranges(int tiles, int m, const Key* __restrict__ tkey,
	int2* __restrict__ ranges)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= tiles) return;
	int bounds[2];
	for (int h = 0; h < 2; ++h) {
		const unsigned int want = (unsigned int)(t + h);
		int lo = 0, hi = m;
		while (lo < hi) {
			const int mid = (lo + hi) >> 1;
			if ((unsigned int)tkey[mid] < want) lo = mid + 1;
			else hi = mid;
		}
		bounds[h] = lo;
	}
	ranges[t] = make_int2(bounds[0], bounds[1]);
}

// Launch order of the compositing blocks: tiles by list length, longest first, in
// power-of-two classes (the order inside a class is free: it changes no result).
// One block.
__global__ void __launch_bounds__(1024) k_tile_order(int tiles, const int2* __restrict__ ranges,
	int* __restrict__ order)
{
	__shared__ int s_count[33], s_start[33];
	if (threadIdx.x < 33) s_count[threadIdx.x] = 0;
	__syncthreads();
	for (int t = threadIdx.x; t < tiles; t += blockDim.x) {
		const int2 r = ranges[t];
		const int len = r.y - r.x;
		atomicAdd(&s_count[len > 0 ? 32 - __clz(len) : 0], 1);
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		int at = 0;
		for (int c = 32; c >= 0; --c) {
			s_start[c] = at;
			at += s_count[c];
		}
	}
	__syncthreads();
	for (int t = threadIdx.x; t < tiles; t += blockDim.x) {
		const int2 r = ranges[t];
		const int len = r.y - r.x;
		order[atomicAdd(&s_start[len > 0 ? 32 - __clz(len) : 0], 1)] = t;
	}
}

// False when the Gaussian (c = centre x, y and the half widths of its alpha >= 1/255
// box) cannot reach alpha 1/255 at any pixel centre of [x0, x1] x [y0, y1]: the
// rectangle's nearest point is outside the box.  Conservative by construction of the
// half widths.
__device__ __forceinline__ bool splat_reaches(float4 c, float x0, float x1, float y0, float y1)
{
	const float nx = fminf(fmaxf(c.x, x0), x1), ny = fminf(fmaxf(c.y, y0), y1);
	return fabsf(c.x - nx) <= c.z && fabsf(c.y - ny) <= c.w;
}

// Front-to-back state of one pixel (renderCUDA's per-thread registers).
struct PixelAcc {
	float T = 1.0f, r = 0.0f, g = 0.0f, b = 0.0f;
	int last = 0, picked = -1;
	bool done = false;
};

// Writes one pixel: colour over the background (or the checker floor where it shows),
// transmittance, contributor count and picked Gaussian.
__device__ __forceinline__ void splat_finish(const RenderFrame& F, int px, int py, const PixelAcc& P,
	float* __restrict__ out, float* __restrict__ final_T, int* __restrict__ n_contrib, int* __restrict__ pick)
{
	const size_t pix = (size_t)py * F.W + px, plane = (size_t)F.W * F.H;
	const float fx = (float)px, fy = (float)py;
	final_T[pix] = P.T;
	n_contrib[pix] = P.last;
	float bgc[3] = { F.bg[0], F.bg[1], F.bg[2] };
	if (F.floor_on && P.T > (1.0f / 255.0f) && F.fl_camh > 0.0f) {
		// ray through the pixel against the ground plane; checker cells faded with distance
		const float ndcx = (2.0f * fx + 1.0f) / (float)F.W - 1.0f;
		const float ndcy = (2.0f * fy + 1.0f) / (float)F.H - 1.0f;
		const float rx = F.fl_rx[0] * ndcx + F.fl_ry[0] * ndcy + F.fl_rz[0];
		const float ry = F.fl_rx[1] * ndcx + F.fl_ry[1] * ndcy + F.fl_rz[1];
		const float rz = F.fl_rx[2] * ndcx + F.fl_ry[2] * ndcy + F.fl_rz[2];
		const float denom = F.fl_n[0] * rx + F.fl_n[1] * ry + F.fl_n[2] * rz;
		if (denom < -1e-6f) {
			const float s = -F.fl_camh / denom;
			const float ox = F.fl_cam[0] + s * rx - F.fl_origin[0];
			const float oy = F.fl_cam[1] + s * ry - F.fl_origin[1];
			const float oz = F.fl_cam[2] + s * rz - F.fl_origin[2];
			const float fade = expf(-(ox * ox + oy * oy + oz * oz) * F.fl_inv_fade2);
			if (fade > (1.0f / 255.0f)) {
				const float u = ox * F.fl_t1[0] + oy * F.fl_t1[1] + oz * F.fl_t1[2];
				const float v = ox * F.fl_t2[0] + oy * F.fl_t2[1] + oz * F.fl_t2[2];
				const int parity = ((int)floorf(u) + (int)floorf(v)) & 1;
				const float dl2 = rx * rx + ry * ry + rz * rz;
				const float blur = fminf(1.0f, s * dl2 * F.fl_pix / (-denom));
				const float shade = (parity ? 1.0f : 0.0f) * (1.0f - blur) + 0.5f * blur;
				const float fc = 0.50f + 0.32f * shade;
				for (int ch = 0; ch < 3; ++ch) bgc[ch] += (fc - bgc[ch]) * fade;
			}
		}
	}
	out[pix] = P.r + P.T * bgc[0];
	out[plane + pix] = P.g + P.T * bgc[1];
	out[2 * plane + pix] = P.b + P.T * bgc[2];
	if (F.pick && P.picked != -1) pick[pix] = P.picked;
}

// One block of 256 threads per 16x16 tile, tiles launched longest list first
// (tile_order): warp w owns the 8x4 region ((w % 2) * 8, (w / 2) * 4), one pixel per
// lane, and the eight warps run without block barriers (their reads of the tile's list
// meet in the SM's L1).  A warp walks the tile's list 64 entries a step, two per lane,
// software-pipelined: the list indices of step s + 2 and the centre, conic and colour
// of step s + 1 are in flight while step s is tested and blended, so the dependent
// index -> Gaussian gathers of a long list do not serialise.  Each entry is tested
// against the warp's region (splat_reaches: the box outside which its alpha stays
// below 1/255, computed in k_splat_prepare); survivors are packed into the warp's
// shared-memory slots with their list position and the pixels visit them in list
// order, two Gaussians per iteration (their alphas are independent of T).  A Gaussian
// left out would have been skipped at each of the region's pixels and the position is
// carried along, so colour, transmittance, contributor count and pick equal those of
// the full list.
constexpr int kTileThreads = 256;
constexpr int kSpan = 64;

struct SplatEntry {
	int g;
	float4 c;
	float4 co, col;
};

__device__ __forceinline__ void splat_fetch(SplatEntry& e, int g, const float4* __restrict__ xy,
	const float4* __restrict__ conic_op, const float4* __restrict__ rgb)
{
	e.g = g;
	e.c = xy[g];
	e.co = conic_op[g];
	e.col = rgb[g];
}

// alpha of a Gaussian at a pixel, or 0 where renderCUDA skips it (power > 0 or
// alpha < 1/255)
__device__ __forceinline__ float splat_alpha(float fx, float fy, float2 c, float4 co)
{
	const float dx = c.x - fx, dy = c.y - fy;
	const float power = -0.5f * (co.x * dx * dx + co.z * dy * dy) - co.y * dx * dy;
	if (power > 0.0f) return 0.0f;
	const float alpha = fminf(0.99f, co.w * expf(power));
	return alpha < 1.0f / 255.0f ? 0.0f : alpha;
}

// Front-to-back step of one pixel over one Gaussian (renderCUDA's inner loop): stop
// before T drops below 1e-4, otherwise accumulate colour and record the contributor's
// list position.
__device__ __forceinline__ void splat_apply(PixelAcc& P, float alpha, float4 col, int id, int rank, bool pick_on)
{
	if (P.done || alpha == 0.0f) return;
	if (pick_on && P.picked == -1 && alpha > 0.1f) P.picked = id;
	const float tn = P.T * (1.0f - alpha);
	if (tn < 0.0001f) { P.done = true; return; }
	const float w = alpha * P.T;
	P.r += col.x * w;
	P.g += col.y * w;
	P.b += col.z * w;
	P.T = tn;
	P.last = rank + 1;
}

__global__ void __launch_bounds__(kTileThreads, 3) k_splat_tiles(RenderFrame F, const int* __restrict__ tile_order,
	const int2* __restrict__ ranges, const int* __restrict__ val, const float4* __restrict__ xy,
	const float4* __restrict__ conic_op, const float4* __restrict__ rgb, float* __restrict__ out,
	float* __restrict__ final_T, int* __restrict__ n_contrib, int* __restrict__ pick)
{
	constexpr int kWarps = kTileThreads / 32;
	__shared__ float4 s_co[kWarps][kSpan], s_rgb[kWarps][kSpan];
	__shared__ float2 s_xy[kWarps][kSpan];
	__shared__ int s_id[kWarps][kSpan], s_rank[kWarps][kSpan];
	const int tile = tile_order[blockIdx.x];
	const int bx = tile % F.tiles_x, by = tile / F.tiles_x;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int qx = bx * kTile + (warp & 1) * 8, qy = by * kTile + (warp >> 1) * 4;
	const int qx1 = min(qx + 7, F.W - 1), qy1 = min(qy + 3, F.H - 1);
	const int px = qx + (lane & 7), py = qy + (lane >> 3);
	const bool inside = px < F.W && py < F.H;
	const float fx = (float)px, fy = (float)py;
	const float rx0 = (float)qx, rx1 = (float)qx1, ry0 = (float)qy, ry1 = (float)qy1;
	const bool pick_on = F.pick != 0;
	PixelAcc A;
	A.done = !inside;
	if (qx <= qx1 && qy <= qy1) {
		const int2 r = ranges[tile];
		SplatEntry cur[2], nxt[2];
		int nv[2];
		// prologue: step 0 gathered, step 1 indices loaded
#pragma unroll
		for (int e = 0; e < 2; ++e) {
			const int k = r.x + lane + 32 * e;
			cur[e].g = -1;
			if (k < r.y) splat_fetch(cur[e], val[k], xy, conic_op, rgb);
			nv[e] = k + kSpan < r.y ? val[k + kSpan] : -1;
		}
		for (int base = r.x; base < r.y; base += kSpan) {
			if (__all_sync(0xffffffffu, A.done)) break;
			// in flight: gathers of step + 1, indices of step + 2
#pragma unroll
			for (int e = 0; e < 2; ++e) {
				nxt[e].g = -1;
				if (nv[e] >= 0) splat_fetch(nxt[e], nv[e], xy, conic_op, rgb);
				const int k2 = base + lane + 32 * e + 2 * kSpan;
				nv[e] = k2 < r.y ? val[k2] : -1;
			}
			bool keep[2];
#pragma unroll
			for (int e = 0; e < 2; ++e)
				keep[e] = cur[e].g >= 0 && splat_reaches(cur[e].c, rx0, rx1, ry0, ry1);
			const unsigned b0 = __ballot_sync(0xffffffffu, keep[0]);
			const unsigned b1 = __ballot_sync(0xffffffffu, keep[1]);
			const unsigned lt = (1u << lane) - 1u;
#pragma unroll
			for (int e = 0; e < 2; ++e)
				if (keep[e]) {
					const int at = e == 0 ? __popc(b0 & lt) : __popc(b0) + __popc(b1 & lt);
					s_xy[warp][at] = make_float2(cur[e].c.x, cur[e].c.y);
					s_co[warp][at] = cur[e].co;
					s_rgb[warp][at] = cur[e].col;
					s_id[warp][at] = cur[e].g;
					s_rank[warp][at] = base - r.x + lane + 32 * e;
				}
			__syncwarp();
			const int kept = __popc(b0) + __popc(b1);
			int j = 0;
			for (; j + 1 < kept && !A.done; j += 2) {
				const float a0 = splat_alpha(fx, fy, s_xy[warp][j], s_co[warp][j]);
				const float a1 = splat_alpha(fx, fy, s_xy[warp][j + 1], s_co[warp][j + 1]);
				splat_apply(A, a0, s_rgb[warp][j], s_id[warp][j], s_rank[warp][j], pick_on);
				splat_apply(A, a1, s_rgb[warp][j + 1], s_id[warp][j + 1], s_rank[warp][j + 1], pick_on);
			}
			if (j < kept && !A.done)
				splat_apply(A, splat_alpha(fx, fy, s_xy[warp][j], s_co[warp][j]), s_rgb[warp][j], s_id[warp][j],
					s_rank[warp][j], pick_on);
			__syncwarp();
#pragma unroll
			for (int e = 0; e < 2; ++e) cur[e] = nxt[e];
		}
	}
	if (inside) splat_finish(F, px, py, A, out, final_T, n_contrib, pick);
}

}  // namespace dev
}  // namespace xpbd
