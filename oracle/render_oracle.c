/* CPU restatement of the viewer's 3DGS forward rasteriser (test infrastructure only:
 * the parity checker of the library's splatting pass, never a product path).
 *
 * Follows the reference as compiled into its viewer:
 *   preprocess   preprocessCUDA (forward.cu:1919-2467) with the demo modes off (no
 *                wave / twist / bubble, pivot and covariance rotations 0): in_frustum
 *                (auxiliary.h:152-177), crop box (forward.cu:2006-2008), ndc2Pix
 *                (auxiliary.h:41-44, in double), computeCov3D (forward.cu:903-938),
 *                computeCov2D (forward.cu:701-790), low-pass 0.3 and antialiasing
 *                scale (forward.cu:2343-2354), radius and getRect (forward.cu:2366-2394,
 *                auxiliary.h:46-56), computeColorFromSH (forward.cu:638-698)
 *   binning      duplicateWithKeys / cub radix sort / identifyTileRanges
 *                (rasterizer_impl.cu:64-140, 330-370): pairs in Gaussian order, keyed
 *                (tile << 32 | depth bits), stable-sorted
 *   compositing  renderCUDA (forward.cu:2469-2650): front-to-back, alpha = min(0.99,
 *                o exp(power)), skip alpha < 1/255, stop when T would drop below 1e-4,
 *                picking (first alpha > 0.1), checker floor in place of the background
 * Arithmetic is FP32 in the library kernel's order (products and sums rounded one at a
 * time: the file is compiled with -ffp-contract=off).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "xpbd_oracle.h"

#define TILE 16

typedef struct {
	uint64_t key;
	int g;
	long long gen;   /* generation order: the stable-sort tie break */
} Pair;

static int pair_cmp(const void* a, const void* b)
{
	const Pair* x = (const Pair*)a;
	const Pair* y = (const Pair*)b;
	if (x->key != y->key) return x->key < y->key ? -1 : 1;
	return (x->gen > y->gen) - (x->gen < y->gen);
}

static void sh_rgb(int deg, const float* c, float x, float y, float z, float out[3])
{
	const float c0 = 0.28209479177387814f, c1 = 0.4886025119029199f;
	for (int ch = 0; ch < 3; ++ch) {
		float r = c0 * c[ch];
		if (deg > 0) {
			r = r - c1 * y * c[3 + ch] + c1 * z * c[6 + ch] - c1 * x * c[9 + ch];
			if (deg > 1) {
				const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
				const float w2[5] = { 1.0925484305920792f * xy, -1.0925484305920792f * yz,
					0.31539156525252005f * (2.0f * zz - xx - yy), -1.0925484305920792f * xz,
					0.5462742152960396f * (xx - yy) };
				for (int k = 0; k < 5; ++k) r += w2[k] * c[3 * (4 + k) + ch];
				if (deg > 2) {
					const float w3[7] = { -0.5900435899266435f * y * (3.0f * xx - yy), 2.890611442640554f * xy * z,
						-0.4570457994644658f * y * (4.0f * zz - xx - yy),
						0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy),
						-0.4570457994644658f * x * (4.0f * zz - xx - yy), 1.445305721320277f * z * (xx - yy),
						-0.5900435899266435f * x * (xx - 3.0f * yy) };
					for (int k = 0; k < 7; ++k) r += w3[k] * c[3 * (9 + k) + ch];
				}
			}
		}
		out[ch] = fmaxf(r + 0.5f, 0.0f);
	}
}

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

long long oracle_render(int n, const float* pos, const float* scales, const float* quats, const float* opacity,
	const float* colors, int sh_degree, const float* V, const float* P, const float* campos, int W, int H,
	float tan_fovx, float tan_fovy, float scale_mod, int antialias, const float* box_lo, const float* box_hi,
	const float* bg, int pick, const float* floor_p, float* out, float* final_T, int* n_contrib, int* picked,
	int* radii_out)
{
	if (n < 0 || W <= 0 || H <= 0) return -1;
	const int tx_n = (W + TILE - 1) / TILE, ty_n = (H + TILE - 1) / TILE, tiles = tx_n * ty_n;
	const float focal_x = W / (2.0f * tan_fovx), focal_y = H / (2.0f * tan_fovy);
	const int coeffs = sh_degree < 0 ? 1 : (sh_degree + 1) * (sh_degree + 1);
	float* xy = (float*)malloc(sizeof(float) * 2 * (size_t)(n ? n : 1));
	float* co = (float*)malloc(sizeof(float) * 4 * (size_t)(n ? n : 1));
	float* rgb = (float*)malloc(sizeof(float) * 3 * (size_t)(n ? n : 1));
	float* depth = (float*)malloc(sizeof(float) * (size_t)(n ? n : 1));
	int* rect = (int*)malloc(sizeof(int) * 4 * (size_t)(n ? n : 1));
	int* touched = (int*)calloc((size_t)(n ? n : 1), sizeof(int));
	long long total = 0;
	for (int i = 0; i < n; ++i) {
		if (radii_out) radii_out[i] = 0;
		const float px3 = pos[3 * i], py3 = pos[3 * i + 1], pz3 = pos[3 * i + 2];
		const float vx = V[0] * px3 + V[4] * py3 + V[8] * pz3 + V[12];
		const float vy = V[1] * px3 + V[5] * py3 + V[9] * pz3 + V[13];
		const float vz = V[2] * px3 + V[6] * py3 + V[10] * pz3 + V[14];
		if (vz <= 0.2f) continue;
		if (box_lo && box_hi &&
			(px3 < box_lo[0] || py3 < box_lo[1] || pz3 < box_lo[2] || px3 > box_hi[0] || py3 > box_hi[1] ||
				pz3 > box_hi[2]))
			continue;
		const float hx = P[0] * px3 + P[4] * py3 + P[8] * pz3 + P[12];
		const float hy = P[1] * px3 + P[5] * py3 + P[9] * pz3 + P[13];
		const float hw = P[3] * px3 + P[7] * py3 + P[11] * pz3 + P[15];
		const float iw = 1.0f / (hw + 0.0000001f);
		const float px = (float)((((double)(hx * iw) + 1.0) * W - 1.0) * 0.5);
		const float py = (float)((((double)(hy * iw) + 1.0) * H - 1.0) * 0.5);
		const float qr = quats[4 * i], qx = quats[4 * i + 1], qy = quats[4 * i + 2], qz = quats[4 * i + 3];
		const float R[3][3] = { { 1.f - 2.f * (qy * qy + qz * qz), 2.f * (qx * qy - qr * qz), 2.f * (qx * qz + qr * qy) },
			{ 2.f * (qx * qy + qr * qz), 1.f - 2.f * (qx * qx + qz * qz), 2.f * (qy * qz - qr * qx) },
			{ 2.f * (qx * qz - qr * qy), 2.f * (qy * qz + qr * qx), 1.f - 2.f * (qx * qx + qy * qy) } };
		const float s[3] = { scale_mod * scales[3 * i], scale_mod * scales[3 * i + 1], scale_mod * scales[3 * i + 2] };
		float M[3][3];
		for (int c = 0; c < 3; ++c)
			for (int r = 0; r < 3; ++r) M[r][c] = s[r] * R[c][r];
		float S[3][3];
		for (int a = 0; a < 3; ++a)
			for (int b = a; b < 3; ++b) S[a][b] = S[b][a] = M[0][a] * M[0][b] + M[1][a] * M[1][b] + M[2][a] * M[2][b];
		const float limx = 1.3f * tan_fovx, limy = 1.3f * tan_fovy;
		const float tx = fminf(limx, fmaxf(-limx, vx / vz)) * vz;
		const float ty = fminf(limy, fmaxf(-limy, vy / vz)) * vz;
		const float j00 = focal_x / vz, j02 = -(focal_x * tx) / (vz * vz);
		const float j11 = focal_y / vz, j12 = -(focal_y * ty) / (vz * vz);
		float T0[3], T1[3];
		for (int c = 0; c < 3; ++c) {
			T0[c] = j00 * V[4 * c] + j02 * V[4 * c + 2];
			T1[c] = j11 * V[4 * c + 1] + j12 * V[4 * c + 2];
		}
		float u0[3], u1[3];
		for (int a = 0; a < 3; ++a) {
			u0[a] = S[a][0] * T0[0] + S[a][1] * T0[1] + S[a][2] * T0[2];
			u1[a] = S[a][0] * T1[0] + S[a][1] * T1[1] + S[a][2] * T1[2];
		}
		float ca = T0[0] * u0[0] + T0[1] * u0[1] + T0[2] * u0[2];
		const float cb = T0[0] * u1[0] + T0[1] * u1[1] + T0[2] * u1[2];
		float cc = T1[0] * u1[0] + T1[1] * u1[1] + T1[2] * u1[2];
		const float det0 = ca * cc - cb * cb;
		ca += 0.3f;
		cc += 0.3f;
		const float det = ca * cc - cb * cb;
		const float aa = antialias ? sqrtf(fmaxf(0.000025f, det0 / det)) : 1.0f;
		if (det == 0.0f) continue;
		const float idet = 1.0f / det;
		const float mid = 0.5f * (ca + cc);
		const float l1 = mid + sqrtf(fmaxf(0.1f, mid * mid - det));
		const float l2 = mid - sqrtf(fmaxf(0.1f, mid * mid - det));
		const int radius = (int)ceilf(3.0f * sqrtf(fmaxf(l1, l2)));
		const int x0 = imin(tx_n, imax(0, (int)((px - radius) / TILE)));
		const int y0 = imin(ty_n, imax(0, (int)((py - radius) / TILE)));
		const int x1 = imin(tx_n, imax(0, (int)((px + radius + TILE - 1) / TILE)));
		const int y1 = imin(ty_n, imax(0, (int)((py + radius + TILE - 1) / TILE)));
		const int cnt = (x1 - x0) * (y1 - y0);
		if (cnt == 0) continue;
		if (sh_degree >= 0) {
			float dx = px3 - campos[0], dy = py3 - campos[1], dz = pz3 - campos[2];
			const float len = sqrtf(dx * dx + dy * dy + dz * dz);
			dx /= len; dy /= len; dz /= len;
			sh_rgb(sh_degree, colors + (size_t)3 * coeffs * i, dx, dy, dz, rgb + 3 * i);
		} else {
			rgb[3 * i] = colors[3 * i]; rgb[3 * i + 1] = colors[3 * i + 1]; rgb[3 * i + 2] = colors[3 * i + 2];
		}
		xy[2 * i] = px; xy[2 * i + 1] = py;
		co[4 * i] = cc * idet; co[4 * i + 1] = -cb * idet; co[4 * i + 2] = ca * idet; co[4 * i + 3] = opacity[i] * aa;
		depth[i] = vz;
		rect[4 * i] = x0; rect[4 * i + 1] = y0; rect[4 * i + 2] = x1; rect[4 * i + 3] = y1;
		touched[i] = cnt;
		if (radii_out) radii_out[i] = radius;
		total += cnt;
	}
	/* pairs in Gaussian order, stable sort by (tile, depth) */
	Pair* pairs = (Pair*)malloc(sizeof(Pair) * (size_t)(total ? total : 1));
	long long at = 0;
	for (int i = 0; i < n; ++i) {
		if (!touched[i]) continue;
		uint32_t dbits;
		memcpy(&dbits, &depth[i], 4);
		for (int y = rect[4 * i + 1]; y < rect[4 * i + 3]; ++y)
			for (int x = rect[4 * i]; x < rect[4 * i + 2]; ++x) {
				pairs[at].key = ((uint64_t)(uint32_t)(y * tx_n + x) << 32) | dbits;
				pairs[at].g = i;
				pairs[at].gen = at;
				++at;
			}
	}
	qsort(pairs, (size_t)total, sizeof(Pair), pair_cmp);
	long long* start = (long long*)malloc(sizeof(long long) * (size_t)(tiles + 1));
	{
		long long k = 0;
		for (int t = 0; t <= tiles; ++t) {
			while (k < total && (long long)(pairs[k].key >> 32) < t) ++k;
			start[t] = k;
		}
	}
	/* floor (renderCUDA's ground composite) */
	int floor_on = 0;
	float fl_rx[3] = { 0 }, fl_ry[3] = { 0 }, fl_rz[3] = { 0 }, fl_n[3] = { 0 }, fl_t1[3] = { 0 }, fl_t2[3] = { 0 },
		fl_o[3] = { 0 }, fl_camh = 0, fl_pix = 0, fl_if2 = 0;
	if (floor_p) {
		floor_on = 1;
		for (int k = 0; k < 3; ++k) fl_n[k] = floor_p[k];
		float a[3] = { 0, 0, 0 };
		const float ax = fabsf(fl_n[0]), ay = fabsf(fl_n[1]), az = fabsf(fl_n[2]);
		a[(ax <= ay && ax <= az) ? 0 : (ay <= az ? 1 : 2)] = 1.0f;
		const float d = a[0] * fl_n[0] + a[1] * fl_n[1] + a[2] * fl_n[2];
		float x = a[0] - d * fl_n[0], y = a[1] - d * fl_n[1], z = a[2] - d * fl_n[2];
		const float len = sqrtf(x * x + y * y + z * z);
		if (len > 1e-12f) { x /= len; y /= len; z /= len; }
		const float t1[3] = { x, y, z };
		const float t2[3] = { fl_n[1] * z - fl_n[2] * y, fl_n[2] * x - fl_n[0] * z, fl_n[0] * y - fl_n[1] * x };
		const float inv_checker = 1.0f / fmaxf(floor_p[7], 1e-8f);
		for (int k = 0; k < 3; ++k) {
			fl_rx[k] = V[4 * k] * tan_fovx;
			fl_ry[k] = V[4 * k + 1] * tan_fovy;
			fl_rz[k] = V[4 * k + 2];
			fl_t1[k] = t1[k] * inv_checker;
			fl_t2[k] = t2[k] * inv_checker;
			fl_o[k] = floor_p[4 + k];
		}
		fl_camh = fl_n[0] * campos[0] + fl_n[1] * campos[1] + fl_n[2] * campos[2] - floor_p[3];
		fl_pix = 2.0f * tan_fovy / (float)H * inv_checker;
		const float fade = fmaxf(floor_p[8], 1e-8f);
		fl_if2 = 1.0f / fmaxf(fade * fade, 1e-12f);
	}
	const size_t plane = (size_t)W * H;
	for (int py_i = 0; py_i < H; ++py_i)
		for (int px_i = 0; px_i < W; ++px_i) {
			const int tile = (py_i / TILE) * tx_n + px_i / TILE;
			const float fx = (float)px_i, fy = (float)py_i;
			float T = 1.0f, c[3] = { 0, 0, 0 };
			int contributor = 0, last = 0, pk = -1;
			for (long long k = start[tile]; k < start[tile + 1]; ++k) {
				++contributor;
				const int g = pairs[k].g;
				const float dx = xy[2 * g] - fx, dy = xy[2 * g + 1] - fy;
				const float* q = co + 4 * g;
				const float power = -0.5f * (q[0] * dx * dx + q[2] * dy * dy) - q[1] * dx * dy;
				if (power > 0.0f) continue;
				const float alpha = fminf(0.99f, q[3] * expf(power));
				if (alpha < 1.0f / 255.0f) continue;
				if (pick && pk == -1 && alpha > 0.1f) pk = g;
				const float tn = T * (1.0f - alpha);
				if (tn < 0.0001f) break;
				const float w = alpha * T;
				for (int ch = 0; ch < 3; ++ch) c[ch] += rgb[3 * g + ch] * w;
				T = tn;
				last = contributor;
			}
			const size_t pix = (size_t)py_i * W + px_i;
			float bgc[3] = { bg ? bg[0] : 0.0f, bg ? bg[1] : 0.0f, bg ? bg[2] : 0.0f };
			if (floor_on && T > (1.0f / 255.0f) && fl_camh > 0.0f) {
				const float ndcx = (2.0f * fx + 1.0f) / (float)W - 1.0f;
				const float ndcy = (2.0f * fy + 1.0f) / (float)H - 1.0f;
				const float rx = fl_rx[0] * ndcx + fl_ry[0] * ndcy + fl_rz[0];
				const float ry = fl_rx[1] * ndcx + fl_ry[1] * ndcy + fl_rz[1];
				const float rz = fl_rx[2] * ndcx + fl_ry[2] * ndcy + fl_rz[2];
				const float denom = fl_n[0] * rx + fl_n[1] * ry + fl_n[2] * rz;
				if (denom < -1e-6f) {
					const float sd = -fl_camh / denom;
					const float ox = campos[0] + sd * rx - fl_o[0];
					const float oy = campos[1] + sd * ry - fl_o[1];
					const float oz = campos[2] + sd * rz - fl_o[2];
					const float fade = expf(-(ox * ox + oy * oy + oz * oz) * fl_if2);
					if (fade > (1.0f / 255.0f)) {
						const float u = ox * fl_t1[0] + oy * fl_t1[1] + oz * fl_t1[2];
						const float v = ox * fl_t2[0] + oy * fl_t2[1] + oz * fl_t2[2];
						const int parity = ((int)floorf(u) + (int)floorf(v)) & 1;
						const float dl2 = rx * rx + ry * ry + rz * rz;
						const float blur = fminf(1.0f, sd * dl2 * fl_pix / (-denom));
						const float shade = (parity ? 1.0f : 0.0f) * (1.0f - blur) + 0.5f * blur;
						const float fc = 0.50f + 0.32f * shade;
						for (int ch = 0; ch < 3; ++ch) bgc[ch] += (fc - bgc[ch]) * fade;
					}
				}
			}
			for (int ch = 0; ch < 3; ++ch) out[ch * plane + pix] = c[ch] + T * bgc[ch];
			if (final_T) final_T[pix] = T;
			if (n_contrib) n_contrib[pix] = last;
			if (picked) picked[pix] = pick ? pk : -1;
		}
	free(start);
	free(pairs);
	free(xy); free(co); free(rgb); free(depth); free(rect); free(touched);
	return total;
}
