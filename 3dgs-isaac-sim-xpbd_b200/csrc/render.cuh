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
	const float* __restrict__ colors, float2* __restrict__ xy, float4* __restrict__ conic_op,
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
		col = sh_color(F.sh_deg, colors + (size_t)3 * F.sh_coeffs * i, make_float3(dx, dy, dz));
	} else {
		col = make_float3(colors[3 * i], colors[3 * i + 1], colors[3 * i + 2]);
	}
	xy[i] = make_float2(px, py);
	conic_op[i] = make_float4(cc * idet, -cb * idet, ca * idet, opacity[i] * aa);
	rgb[i] = make_float4(col.x, col.y, col.z, 0.0f);
	dkey[i] = __float_as_uint(vz);   // positive floats order as unsigned integers
	radii[i] = radius;
	rect[i] = make_int4(x0, y0, x1, y1);
	touched[i] = cnt;
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

// one (tile, Gaussian) pair per touched tile, Gaussians in depth order
__global__ void __launch_bounds__(kBlock) k_splat_pairs(int n, const int* __restrict__ order,
	const long long* __restrict__ offs, const int4* __restrict__ rect, int tiles_x, unsigned int* __restrict__ tkey,
	int* __restrict__ val)
{
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= n) return;
	long long at = offs[k];
	if (offs[k + 1] == at) return;
	const int g = order[k];
	const int4 r = rect[g];
	for (int y = r.y; y < r.w; ++y)
		for (int x = r.x; x < r.z; ++x) {
			tkey[at] = (unsigned int)(y * tiles_x + x);
			val[at] = g;
			++at;
		}
}

// [start, end) of every tile in the sorted pair list (ranges zeroed before)
__global__ void __launch_bounds__(kBlock) k_splat_ranges(int m, const unsigned int* __restrict__ tkey,
	int2* __restrict__ ranges)
{
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= m) return;
	const unsigned int tile = tkey[t];
	if (t == 0 || tkey[t - 1] != tile) ranges[tile].x = t;
	if (t == m - 1 || tkey[t + 1] != tile) ranges[tile].y = t + 1;
}

// One block per 16x16 tile, one thread per pixel.
__global__ void __launch_bounds__(kTilePix) k_splat_tiles(RenderFrame F, const int2* __restrict__ ranges,
	const int* __restrict__ val, const float2* __restrict__ xy, const float4* __restrict__ conic_op,
	const float4* __restrict__ rgb, float* __restrict__ out, float* __restrict__ final_T,
	int* __restrict__ n_contrib, int* __restrict__ pick)
{
	__shared__ int s_id[kTilePix];
	__shared__ float2 s_xy[kTilePix];
	__shared__ float4 s_co[kTilePix];
	const int tile = blockIdx.y * F.tiles_x + blockIdx.x;
	const int pxi = blockIdx.x * kTile + (int)threadIdx.x % kTile;
	const int pyi = blockIdx.y * kTile + (int)threadIdx.x / kTile;
	const bool inside = pxi < F.W && pyi < F.H;
	const float fx = (float)pxi, fy = (float)pyi;
	const int2 r = ranges[tile];
	float T = 1.0f;
	float cr = 0.0f, cg = 0.0f, cbl = 0.0f;
	int contributor = 0, last = 0, picked = -1;
	bool done = !inside;
	int todo = r.y - r.x;
	for (int base = r.x; base < r.y; base += kTilePix, todo -= kTilePix) {
		if (__syncthreads_count(done) == kTilePix) break;
		const int k = base + (int)threadIdx.x;
		if (k < r.y) {
			const int g = val[k];
			s_id[threadIdx.x] = g;
			s_xy[threadIdx.x] = xy[g];
			s_co[threadIdx.x] = conic_op[g];
		}
		__syncthreads();
		const int cnt = min(kTilePix, todo);
		for (int j = 0; !done && j < cnt; ++j) {
			++contributor;
			const float2 c = s_xy[j];
			const float4 co = s_co[j];
			const float dx = c.x - fx, dy = c.y - fy;
			const float power = -0.5f * (co.x * dx * dx + co.z * dy * dy) - co.y * dx * dy;
			if (power > 0.0f) continue;
			const float alpha = fminf(0.99f, co.w * expf(power));
			if (alpha < 1.0f / 255.0f) continue;
			if (F.pick && picked == -1 && alpha > 0.1f) picked = s_id[j];
			const float tn = T * (1.0f - alpha);
			if (tn < 0.0001f) { done = true; continue; }
			const float4 col = rgb[s_id[j]];
			const float w = alpha * T;
			cr += col.x * w;
			cg += col.y * w;
			cbl += col.z * w;
			T = tn;
			last = contributor;
		}
	}
	if (!inside) return;
	const size_t pix = (size_t)pyi * F.W + pxi, plane = (size_t)F.W * F.H;
	final_T[pix] = T;
	n_contrib[pix] = last;
	float bgc[3] = { F.bg[0], F.bg[1], F.bg[2] };
	if (F.floor_on && T > (1.0f / 255.0f) && F.fl_camh > 0.0f) {
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
	out[pix] = cr + T * bgc[0];
	out[plane + pix] = cg + T * bgc[1];
	out[2 * plane + pix] = cbl + T * bgc[2];
	if (F.pick && picked != -1) pick[pix] = picked;
}

}  // namespace dev
}  // namespace xpbd
