/*
 * CPU oracle for the XPBD Gaussian-graph solver step — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C (C11 + OpenMP) restatement of the reference solver's step as reached
 * through its C ABI (native/xpbd_capi.cu -> native/solver_core/cuda_rasterizer/
 * forward.cu).  liboracle.so exports the same 29 `xpbd_*` entry points as the
 * reference library, so one ctypes bridge drives the reference, this oracle and the
 * product library alike.  Each function in xpbd_oracle.c cites the reference
 * file:line it restates.
 *
 * Pinning: the restatement is checked against golden vectors produced by the
 * reference solver itself (the .npz files in tests/golden, made by tests/golden/make_golden.py
 * from oracle/_ref/libxpbd_ref.so): cluster CSR, colourings and self-collision
 * keys / order / candidate lists bit-exactly, positions and shapes within the
 * FP32 tolerances written in the tests.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this
 * library, and only as the checker or the timed CPU baseline.  The product path
 * never links it.
 *
 * Out of the restatement (documented, returns an error or is a no-op): object mode
 * (xpbd_set_object_shape > 0), the squash/press harness and ellipsoid contact shapes.
 */
#ifndef XPBD_ORACLE_H
#define XPBD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Gauss-Seidel toggles (reference forward.cu:3780-3812, not in its C ABI). */
void oracle_set_gs(int distance, int volume);
/* current positions (float3[n], caller order); velocities are kept */
int oracle_set_positions(const float* pos, int n);
/* Volume Kernel A/B shape: 0 auto (warp when mean members >= 40), 1 thread, 2 warp
 * (forward.cu:4043-4060).  The modes differ only in summation order. */
void oracle_set_volume_warp_mode(int mode);
/* Worker threads for the per-Gaussian loops (0 = all cores). */
void oracle_set_threads(int n);
int oracle_get_threads(void);
/* Stage buffers, same names as oracle/ref_shim.cu.  Returns the element count
 * (out == NULL: count only) or -1. */
int oracle_int(const char* name, int* out, long long cap);
int oracle_float(const char* name, float* out, long long cap);
void oracle_sizes(long long* out);
/* The once-per-step self-collision build on given start / predicted positions. */
int oracle_selfcol_build(const float* x, const float* p);
/* ChainMail propagation (forward.cu:12808-13006, dense path): material controls,
 * seeds (move + arrival time 0), prop_iters + relax_iters + 1 sweeps, arrival times. */
void oracle_chainmail_set_material(float global_scale, float air, float skin, float bone, int use_edge_stiffness,
	float edge_influence);
int oracle_chainmail_seed(int count, const int* idx, const float* delta);
int oracle_chainmail_run(int prop_iters, int relax_iters, float prop_strength, float relax_stiffness,
	float relax_damping);
int oracle_chainmail_times(float* out, int n);
/* Stateless 3DGS forward rasteriser (render_oracle.c): explicit positions, scales,
 * quaternions (w, x, y, z), opacities and colours (RGB when sh_degree is -1, else
 * [n][(d+1)^2][3] SH coefficients); camera as the library's xpbd_b200_render; box_lo /
 * box_hi NULL for no crop box; floor_p NULL or {normal[3], height, origin[3], checker,
 * fade radius}.  out is 3 x H x W; final_T, n_contrib, picked (H x W) and radii (n) may
 * be NULL.  Returns the (tile, Gaussian) pair count. */
long long oracle_render(int n, const float* pos, const float* scales, const float* quats, const float* opacity,
	const float* colors, int sh_degree, const float* view, const float* proj, const float* campos, int W, int H,
	float tan_fovx, float tan_fovy, float scale_mod, int antialias, const float* box_lo, const float* box_hi,
	const float* bg, int pick, const float* floor_p, float* out, float* final_T, int* n_contrib, int* picked,
	int* radii);

#ifdef __cplusplus
}
#endif
#endif
