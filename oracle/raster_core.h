/*
 * raster_core.h -- CPU restatement of the reference Gaussian rasterizer
 * (Word2World cudaForwardBackwardRenderer), forward and backward.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle: it is compiled into
 * oracle/liborc_w2w.so and called from tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py.  Nothing in the product links it.
 *
 * The file is included twice by w2w_oracle.c: once with REAL=float (the fp32
 * restatement, bit-for-bit in the reference's operation order) and once with
 * REAL=double (the fp64 re-evaluation of the same algorithm).  Every function
 * cites the reference file:line it restates (paths relative to the reference
 * project root).
 *
 * Floating point: the file is compiled with -ffp-contract=off, so each + - * /
 * is one IEEE rounding and every fused multiply-add is an explicit RFMA().
 * Expressions whose fusion the reference's compiler chose are written through
 * the S2/D2/S3 helpers whose variant index (orc_var[]) selects the pattern;
 * the pinned values are set by the Python wrapper.  Transcendentals (exp, log)
 * are the C library's; the reference's device versions may differ in the last
 * ulp, which the margin outputs below let tests account for.
 */

#ifndef REAL
#error "define REAL before including raster_core.h"
#endif

/* ---- small arithmetic helpers with selectable fusion pattern ------------ */

/* a*b + c*d */
static inline REAL SFX(s2)(int v, REAL a, REAL b, REAL c, REAL d) {
    switch (v) {
    case 1: return RFMA(a, b, c * d);
    case 2: return RFMA(c, d, a * b);
    default: return a * b + c * d;
    }
}
/* a*b - c*d */
static inline REAL SFX(d2)(int v, REAL a, REAL b, REAL c, REAL d) {
    switch (v) {
    case 1: return RFMA(a, b, -(c * d));
    case 2: return RFMA(-c, d, a * b);
    default: return a * b - c * d;
    }
}
/* (a*b + c*d) + e*f */
static inline REAL SFX(s3)(int v, REAL a, REAL b, REAL c, REAL d, REAL e, REAL f) {
    switch (v) {
    case 1: return RFMA(e, f, RFMA(a, b, c * d));
    case 2: return RFMA(e, f, RFMA(c, d, a * b));
    case 3: return RFMA(e, f, a * b + c * d);
    case 4: return RFMA(a, b, c * d) + e * f;
    case 5: return RFMA(c, d, a * b) + e * f;
    case 6: return RFMA(a, b, RFMA(c, d, e * f));
    default: return (a * b + c * d) + e * f;
    }
}
/* a*b + c (single product plus addend) */
static inline REAL SFX(s1)(int v, REAL a, REAL b, REAL c) {
    return v ? RFMA(a, b, c) : a * b + c;
}

/* glm-style mat4 * vec4(p, 1) row r of a column-major 16-float matrix
 * (GLMLibrary/glm/detail/type_mat4x4.inl operator*(mat4, vec4):
 *  (m0*v0 + m1*v1) + (m2*v2 + m3*v3), with v3 == 1). */
static inline REAL SFX(m4row)(int va, int vb, const float* m, int r, REAL x, REAL y, REAL z) {
    REAL a = SFX(s2)(orc_var[va + r], (REAL)m[0 + r], x, (REAL)m[4 + r], y);
    REAL b = SFX(s1)(orc_var[vb + r], (REAL)m[8 + r], z, (REAL)m[12 + r]);
    return a + b;
}

/* ------------------------------------------------------------------------ */
/* Forward: projection  (projection.cu:7-154)                               */
/* ------------------------------------------------------------------------ */
/* Per-Gaussian geometry.  Outputs follow the reference geomBuf fields:
 *   cov3D[6] (projection.cu:60-70), conic_opac[4] (:120-128), means2D[2]
 *   (:142-152), depth = NDC z (:153); plus cov2D[3] and det (covOP/detOP,
 *   :135-136) which the reference keeps in temporaries.
 * Returns 1 if the Gaussian is visible to later stages, 0 if culled by
 * the near test (:75-77) or the determinant test (:116-119).  *clamp_hit is
 * set when the inscribed-circle clamp (:84-89) fires (the reference uses the
 * approximate rsqrtf there, which this restatement cannot reproduce bit for
 * bit; callers treat such Gaussians as outside the bit-exact contract). */
static int SFX(project_one)(const orc_cfg* cfg, const float* mean, const float* scale,
                            const float* q, float opacity,
                            REAL* cov3D, REAL* cov2D, REAL* det_out, REAL* conic_opac,
                            REAL* mean2D, REAL* depth, int* clamp_hit)
{
    const float* V = cfg->view;
    const float* PM = cfg->proj;
    const REAL focal = (REAL)cfg->focal_x;
    const REAL W = (REAL)cfg->W, H = (REAL)cfg->H;
    *clamp_hit = 0;

    /* rotation from quaternion (r, x, y, z) -- projection.cu:43-58 */
    REAL r = q[0], x = q[1], y = q[2], z = q[3];
    REAL xx = x * x, yy = y * y, zz = z * z;
    REAL xy = x * y, xz = x * z, yz = y * z;
    REAL rx = r * x, ry = r * y, rz = r * z;
    (void)xx; (void)yy; (void)zz; (void)xy; (void)xz; (void)yz; (void)rx; (void)ry; (void)rz;
    const int* vq = orc_var + V_RQ; /* one selector per matrix entry, column-major */
    /* columns of the glm matrix before the 0.5 factor */
    REAL Rc[3][3];
    Rc[0][0] = (REAL)2 - (REAL)4 * SFX(s2)(vq[0], y, y, z, z);
    Rc[0][1] = (REAL)4 * SFX(d2)(vq[1], x, y, r, z);
    Rc[0][2] = (REAL)4 * SFX(s2)(vq[2], x, z, r, y);
    Rc[1][0] = (REAL)4 * SFX(s2)(vq[3], x, y, r, z);
    Rc[1][1] = (REAL)2 - (REAL)4 * SFX(s2)(vq[4], x, x, z, z);
    Rc[1][2] = (REAL)4 * SFX(d2)(vq[5], y, z, r, x);
    Rc[2][0] = (REAL)4 * SFX(d2)(vq[6], x, z, r, y);
    Rc[2][1] = (REAL)4 * SFX(s2)(vq[7], y, z, r, x);
    Rc[2][2] = (REAL)2 - (REAL)4 * SFX(s2)(vq[8], x, x, y, y);
    REAL R[3][3];
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 3; ++k) R[c][k] = (REAL)0.5 * Rc[c][k];

    /* Sigma = transpose(R) * transpose(S) * S * R  (projection.cu:60).
     * transpose(R)*S scales column c of R^T by s_c, the second S scales it
     * again; the final product is a full glm mat3 product. */
    REAL s[3] = {scale[0], scale[1], scale[2]};
    REAL A[3][3]; /* A[c][r] = R^T[c][r] * s_c * s_c, R^T[c][r] = R[r][c] */
    for (int c = 0; c < 3; ++c)
        for (int rr = 0; rr < 3; ++rr) A[c][rr] = (R[rr][c] * s[c]) * s[c];
    REAL Sig[3][3];
    /* only the upper triangle is stored (and so computed); selector per stored entry */
    static const int sidx[3][3] = {{0, 1, 2}, {-1, 3, 4}, {-1, -1, 5}};
    for (int c = 0; c < 3; ++c)
        for (int rr = c; rr < 3; ++rr)
            Sig[c][rr] = SFX(s3)(orc_var[V_SIGMA + sidx[c][rr]], A[0][rr], R[c][0], A[1][rr], R[c][1],
                                 A[2][rr], R[c][2]);
    /* packed upper triangle in the reference's order Sigma[i][j], j >= i */
    cov3D[0] = Sig[0][0]; cov3D[1] = Sig[0][1]; cov3D[2] = Sig[0][2];
    cov3D[3] = Sig[1][1]; cov3D[4] = Sig[1][2]; cov3D[5] = Sig[2][2];

    /* view transform (projection.cu:71-77) */
    REAL mx = mean[0], my = mean[1], mz = mean[2];
    REAL tx = SFX(m4row)(V_VIEW_A, V_VIEW_B, V, 0, mx, my, mz);
    REAL ty = SFX(m4row)(V_VIEW_A, V_VIEW_B, V, 1, mx, my, mz);
    REAL tz = SFX(m4row)(V_VIEW_A, V_VIEW_B, V, 2, mx, my, mz);
    REAL tw = SFX(m4row)(V_VIEW_A, V_VIEW_B, V, 3, mx, my, mz);
    tx = tx / tw; ty = ty / tw; tz = tz / tw;
    if (tz <= (REAL)1) return 0;

    /* inscribed-circle clamp (projection.cu:22,78-92).  The reference hard-codes
     * 800 for the image width in camHorizLengthTan; the generic form is W. */
    REAL limit = W / ((REAL)2 * focal);
    REAL rsx = tx / tz, rsy = ty / tz;
    REAL nx = rsx / limit, ny = rsy / limit;
    REAL sq = SFX(s2)(orc_var[V_RAYR2], nx, nx, ny, ny);
    if (sq > (REAL)1) {
        REAL sc = (REAL)1 / RSQRT(sq);
        rsx = rsx * sc; rsy = rsy * sc;
        *clamp_hit = 1;
    }
    tx = rsx * tz;
    ty = rsy * tz;

    /* EWA Jacobian rows (projection.cu:94-101): focal_x on both axes */
    REAL right[3] = {V[0], V[4], V[8]};
    REAL up[3] = {V[1], V[5], V[9]};
    REAL fwd[3] = {V[2], V[6], V[10]};
    REAL zi = (REAL)1 / tz;
    REAL zi2 = zi * zi;
    REAL jx[3], jy[3];
    for (int k = 0; k < 3; ++k) {
        jx[k] = focal * SFX(d2)(orc_var[V_DPROJ + k], right[k], zi, tx * fwd[k], zi2);
        jy[k] = focal * SFX(d2)(orc_var[V_DPROJ + 3 + k], up[k], zi, ty * fwd[k], zi2);
    }
    /* cov2D = [jx.S.jx, jx.S.jy, jy.S.jy]  (projection.cu:102-114) */
    REAL Sm[3][3] = {{cov3D[0], cov3D[1], cov3D[2]},
                     {cov3D[1], cov3D[3], cov3D[4]},
                     {cov3D[2], cov3D[4], cov3D[5]}}; /* column-major, symmetric */
    REAL Sjx[3], Sjy[3];
    for (int rr = 0; rr < 3; ++rr) {
        Sjx[rr] = SFX(s3)(orc_var[V_SIGV + rr], Sm[0][rr], jx[0], Sm[1][rr], jx[1], Sm[2][rr], jx[2]);
        Sjy[rr] = SFX(s3)(orc_var[V_SIGV + 3 + rr], Sm[0][rr], jy[0], Sm[1][rr], jy[1], Sm[2][rr], jy[2]);
    }
    REAL cxx = SFX(s3)(orc_var[V_DOT3 + 0], jx[0], Sjx[0], jx[1], Sjx[1], jx[2], Sjx[2]);
    REAL cxy = SFX(s3)(orc_var[V_DOT3 + 1], jx[0], Sjy[0], jx[1], Sjy[1], jx[2], Sjy[2]);
    REAL cyy = SFX(s3)(orc_var[V_DOT3 + 2], jy[0], Sjy[0], jy[1], Sjy[1], jy[2], Sjy[2]);
    REAL det = SFX(d2)(orc_var[V_DET], cxx, cyy, cxy, cxy);
    if (!(RABS(det) >= (REAL)1e-8f)) return 0;
    REAL dinv = (REAL)1 / det;
    conic_opac[0] = cyy * dinv;
    conic_opac[1] = -cxy * dinv;
    conic_opac[2] = cxx * dinv;
    conic_opac[3] = opacity;
    cov2D[0] = cxx; cov2D[1] = cxy; cov2D[2] = cyy;
    *det_out = det;

    /* screen position and depth through the full projection (projection.cu:142-153) */
    REAL cx = SFX(m4row)(V_PROJ_A, V_PROJ_B, PM, 0, mx, my, mz);
    REAL cy = SFX(m4row)(V_PROJ_A, V_PROJ_B, PM, 1, mx, my, mz);
    REAL cz = SFX(m4row)(V_PROJ_A, V_PROJ_B, PM, 2, mx, my, mz);
    REAL cw = SFX(m4row)(V_PROJ_A, V_PROJ_B, PM, 3, mx, my, mz);
    REAL invW = (REAL)1 / (cw + (REAL)0.00001f);
    REAL ndx = cx * invW, ndy = cy * invW, ndz = cz * invW;
    /* ((ndc + 1) * 0.5) * W - 0.5; patterns 2/3 fuse the NDC multiply into the +1 */
    for (int a = 0; a < 2; ++a) {
        int v = orc_var[V_PIX + a];
        REAL c = a ? cy : cx, nd = a ? ndy : ndx, S = a ? H : W;
        REAL t = (v >= 2) ? RFMA(c, invW, (REAL)1) : nd + (REAL)1;
        t = t * (REAL)0.5;
        mean2D[a] = SFX(s1)(v == 1 || v == 2, t, S, (REAL)-0.5);
    }
    *depth = ndz;
    return 1;
}

/* ------------------------------------------------------------------------ */
/* Forward: ADR culling -- radius and tiles-touched (ADRculling.cu:33-107)  */
/* ------------------------------------------------------------------------ */
/* rect[4] = (xmin, ymin, xmax, ymax) of the allocation rectangle in tiles.
 * margin: smallest relative distance of a value that is floored/truncated/
 * ceiled here from the integer it would flip at (used to explain 1-ulp
 * differences between this restatement's log and the device's). */
static void SFX(adr_one)(const orc_cfg* cfg, const REAL* cov2D, REAL det, const REAL* m2d,
                         float opacity, int* radius, uint32_t* tiles, int* rect, double* margin)
{
    int gw = (cfg->W + 15) / 16, gh = (cfg->H + 15) / 16;
    REAL tr = cov2D[0] + cov2D[2];
    REAL ht = tr * (REAL)0.5;
    REAL dsq = SFX(s1)(orc_var[V_ADR_DELTA], ht, ht, -det);
    REAL root = RSQRT(dsq > (REAL)0.1f ? dsq : (REAL)0.1f);
    REAL y1 = ht + root, y2 = ht - root;
    REAL ymax = y1 > y2 ? y1 : y2;
    REAL allp = (REAL)3 * RSQRT(ymax);
    *margin = 1e30;
    if (!((REAL)opacity > (REAL)0.0039f)) {
        *radius = 0; *tiles = 0; rect[0] = rect[1] = rect[2] = rect[3] = 0;
        return;
    }
    REAL ln = RLOG((REAL)opacity * (REAL)255);
    REAL adapt = RSQRT((REAL)2 * ymax * ln);
    REAL mr = adapt < allp ? adapt : allp;
    *radius = (int)RCEIL(mr);
    REAL vals[4];
    vals[0] = (m2d[0] - mr) / (REAL)16;
    vals[1] = (m2d[1] - mr) / (REAL)16;
    vals[2] = ((m2d[0] + mr) + (REAL)15) / (REAL)16;
    vals[3] = ((m2d[1] + mr) + (REAL)15) / (REAL)16;
    int t[4];
    for (int k = 0; k < 4; ++k) t[k] = (int)vals[k]; /* C truncation == int() */
    {
        double m = 1e30;
        for (int k = 0; k < 4; ++k) {
            double f = (double)vals[k] - floor((double)vals[k]);
            double d = f < 1 - f ? f : 1 - f;
            double rel = d / (fabs((double)vals[k]) + 1e-30);
            if (rel < m) m = rel;
        }
        double fm = (double)mr - floor((double)mr);
        double dm = (fm < 1 - fm ? fm : 1 - fm) / ((double)mr + 1e-30);
        if (dm < m) m = dm;
        *margin = m;
    }
    int x0 = t[0] > 0 ? t[0] : 0, y0 = t[1] > 0 ? t[1] : 0;
    int x1 = t[2] < gw ? t[2] : gw, y1i = t[3] < gh ? t[3] : gh;
    /* An empty rectangle is zero tiles.  (The reference subtracts unsigned
     * values and wraps for Gaussians entirely off the left/top edge; such
     * inputs are outside its defined behaviour.) */
    if (x1 < x0) x1 = x0;
    if (y1i < y0) y1i = y0;
    rect[0] = x0; rect[1] = y0; rect[2] = x1; rect[3] = y1i;
    *tiles = (uint32_t)(x1 - x0) * (uint32_t)(y1i - y0);
}

/* ------------------------------------------------------------------------ */
/* Forward: SH colour (gaussianForwardPass.cu:11-39, 172-263)               */
/* ------------------------------------------------------------------------ */
/* Writes the UNCLAMPED colour (the reference stores resFina, :263) and the
 * per-channel "clamped" flags (colour < 0, :226-253). */
static void SFX(sh_one)(const float* mean, const float* campos, const float* sh, int M, int deg,
                        REAL* rgb, uint8_t* clamped)
{
    REAL v[3] = {(REAL)mean[0] - campos[0], (REAL)mean[1] - campos[1], (REAL)mean[2] - campos[2]};
    int vd = orc_var[V_SH_DOT];
    REAL l2 = SFX(s3)(vd, v[0], v[0], v[1], v[1], v[2], v[2]);
    REAL inv = (REAL)1 / RSQRT(l2);
    REAL x = v[0] * inv, y = v[1] * inv, z = v[2] * inv;
    const float* c = sh;
    int va = orc_var[V_SH_ACC];
    REAL out[3];
    for (int k = 0; k < 3; ++k) out[k] = (REAL)0.28209479177387814f * c[k];
#define ACC(coef, idx) do { REAL _t = (coef); for (int k = 0; k < 3; ++k) out[k] = SFX(s1)(va, _t, (REAL)c[3 * (idx) + k], out[k]); } while (0)
    if (deg >= 1 && M > 3) {
        ACC((REAL)-0.4886025119029199f * y, 1);
        ACC((REAL)0.4886025119029199f * z, 2);
        ACC((REAL)-0.4886025119029199f * x, 3);
    }
    /* polynomial terms; selectors choose which squares are fused into the
     * subtractions (the squares are otherwise rounded products) */
    REAL xx = x * x, yy = y * y, zz = z * z;
    /* k*zz - xx - yy */
    #define KZZ(v, k) ((v) == 1 ? RFMA(-y, y, RFMA(-x, x, (REAL)(k) * zz)) : \
                      (v) == 2 ? RFMA(-y, y, (REAL)(k) * zz - xx) : \
                      (v) == 3 ? RFMA(-x, x, (REAL)(k) * zz) - yy : ((REAL)(k) * zz - xx) - yy)
    /* xx - yy */
    #define XMY(v) ((v) == 1 ? RFMA(x, x, -yy) : (v) == 2 ? RFMA(-y, y, xx) : xx - yy)
    if (deg >= 2 && M > 8) {
        REAL xy = x * y, yz = y * z, xz = x * z;
        ACC((REAL)1.0925484305920792f * xy, 4);
        ACC((REAL)-1.0925484305920792f * yz, 5);
        ACC((REAL)0.3f * KZZ(orc_var[V_SH2A], 2), 6);
        ACC((REAL)-1.0925484305920792f * xz, 7);
        ACC((REAL)0.5462742152960396f * XMY(orc_var[V_SH2B]), 8);
    }
    if (deg >= 3 && M > 15) {
        int v3a = orc_var[V_SH3A], v3c = orc_var[V_SH3C], v3e = orc_var[V_SH3E];
        REAL t9 = v3a == 1 ? RFMA((REAL)3, xx, -yy) : v3a == 2 ? RFMA(-y, y, (REAL)3 * xx) : (REAL)3 * xx - yy;
        REAL t12 = v3c == 1 ? RFMA((REAL)-3, yy, RFMA((REAL)-3, xx, (REAL)2 * zz))
                 : v3c == 2 ? RFMA((REAL)-3, yy, (REAL)2 * zz - (REAL)3 * xx)
                 : v3c == 3 ? RFMA((REAL)-3, xx, (REAL)2 * zz) - (REAL)3 * yy
                            : ((REAL)2 * zz - (REAL)3 * xx) - (REAL)3 * yy;
        REAL t15 = v3e == 1 ? RFMA((REAL)-3, yy, xx) : v3e == 2 ? RFMA(x, x, -((REAL)3 * yy)) : xx - (REAL)3 * yy;
        ACC(((REAL)-0.5900435899266435f * y) * t9, 9);
        ACC((((REAL)2.890611442640554f * x) * y) * z, 10);
        ACC(((REAL)-0.4570457994644658f * y) * KZZ(orc_var[V_SH3B], 4), 11);
        ACC(((REAL)0.3731763325901154f * z) * t12, 12);
        ACC(((REAL)-0.4570457994644658f * x) * KZZ(orc_var[V_SH3B], 4), 13);
        ACC(((REAL)1.445305721320277f * z) * XMY(orc_var[V_SH3D]), 14);
        ACC(((REAL)-0.5900435899266435f * x) * t15, 15);
    }
    #undef KZZ
    #undef XMY
#undef ACC
    for (int k = 0; k < 3; ++k) {
        out[k] = out[k] + (REAL)0.5;
        clamped[k] = out[k] < (REAL)0 ? 1 : 0;
        rgb[k] = out[k];
    }
}

/* Whole per-Gaussian preprocessing for P Gaussians.  Arrays are float32 in
 * both instantiations except the REAL outputs. */
typedef struct {
    const orc_cfg* cfg;
    int P;
    const float* means3D;
    const float* scales;
    const float* rots;
    const float* opac;
    const float* sh;
    REAL* cov3D;
    REAL* cov2D;
    REAL* det;
    REAL* conic_opac;
    REAL* means2D;
    REAL* depth;
    int32_t* radii;
    uint32_t* tiles;
    int32_t* rects;
    REAL* rgb;
    uint8_t* clamped;
    uint8_t* visible;
    uint8_t* clamp_hit;
    double* adr_margin;
} SFX(orc_preprocess_ctx);
static void SFX(orc_preprocess_part)(void* vc_, long long lo_, long long hi_, int tid_)
{
    SFX(orc_preprocess_ctx)* c_ = (SFX(orc_preprocess_ctx)*)vc_;
    const orc_cfg* cfg = c_->cfg;
    (void)c_->P;
    const float* means3D = c_->means3D;
    const float* scales = c_->scales;
    const float* rots = c_->rots;
    const float* opac = c_->opac;
    const float* sh = c_->sh;
    REAL* cov3D = c_->cov3D;
    REAL* cov2D = c_->cov2D;
    REAL* det = c_->det;
    REAL* conic_opac = c_->conic_opac;
    REAL* means2D = c_->means2D;
    REAL* depth = c_->depth;
    int32_t* radii = c_->radii;
    uint32_t* tiles = c_->tiles;
    int32_t* rects = c_->rects;
    REAL* rgb = c_->rgb;
    uint8_t* clamped = c_->clamped;
    uint8_t* visible = c_->visible;
    uint8_t* clamp_hit = c_->clamp_hit;
    double* adr_margin = c_->adr_margin;
    (void)tid_;

    for (int i = (int)lo_; i < (int)hi_; ++i) {
        int ch = 0;
        for (int k = 0; k < 6; ++k) cov3D[6 * i + k] = 0;
        for (int k = 0; k < 4; ++k) conic_opac[4 * i + k] = 0;
        cov2D[3 * i] = cov2D[3 * i + 1] = cov2D[3 * i + 2] = 0;
        det[i] = 0; means2D[2 * i] = means2D[2 * i + 1] = 0; depth[i] = 0;
        int vis = SFX(project_one)(cfg, means3D + 3 * i, scales + 3 * i, rots + 4 * i, opac[i],
                                   cov3D + 6 * i, cov2D + 3 * i, det + i, conic_opac + 4 * i,
                                   means2D + 2 * i, depth + i, &ch);
        visible[i] = (uint8_t)vis;
        clamp_hit[i] = (uint8_t)ch;
        radii[i] = 0; tiles[i] = 0;
        rects[4 * i] = rects[4 * i + 1] = rects[4 * i + 2] = rects[4 * i + 3] = 0;
        adr_margin[i] = 1e30;
        if (vis)
            SFX(adr_one)(cfg, cov2D + 3 * i, det[i], means2D + 2 * i, opac[i], radii + i,
                         tiles + i, rects + 4 * i, adr_margin + i);
        SFX(sh_one)(means3D + 3 * i, cfg->campos, sh + (size_t)i * cfg->M * 3, cfg->M, cfg->degree,
                    rgb + 3 * i, clamped + 3 * i);
    }
}

void SFX(orc_preprocess)(const orc_cfg* cfg, int P,
                         const float* means3D, const float* scales, const float* rots,
                         const float* opac, const float* sh,
                         REAL* cov3D, REAL* cov2D, REAL* det, REAL* conic_opac,
                         REAL* means2D, REAL* depth, int32_t* radii, uint32_t* tiles,
                         int32_t* rects, REAL* rgb, uint8_t* clamped,
                         uint8_t* visible, uint8_t* clamp_hit, double* adr_margin)
{
    SFX(orc_preprocess_ctx) c_ = {cfg, P, means3D, scales, rots, opac, sh, cov3D, cov2D, det, conic_opac, means2D, depth, radii, tiles, rects, rgb, clamped, visible, clamp_hit, adr_margin};
    orc_parallel_for(P, 4096, SFX(orc_preprocess_part), &c_);
}


/* ------------------------------------------------------------------------ */
/* Forward: key emission (prepareSort.cu:178-205, 239-301)                  */
/* ------------------------------------------------------------------------ */
/* offsets: inclusive scan of tiles (gaussianRasterizer.cu:82-117).
 * compat_spill=1 reproduces the reference's emission rectangle
 * (floor/ceil with the integer radius, prepareSort.cu:279-282), which can be
 * larger than the allocation; entries past a Gaussian's allocation overwrite
 * the following Gaussians' slots.  Where several Gaussians write one slot the
 * LOWEST index wins (what a converged warp does: a lower-index thread reaches
 * that slot at a later loop iteration).  Entries at positions >= R are dropped.
 * compat_spill=0 emits exactly the allocation rectangle.
 * Returns the number of entries that fell past R (tail spill). */
long long SFX(orc_emit)(const orc_cfg* cfg, int P, const REAL* means2D, const REAL* depth,
                        const int32_t* radii, const int32_t* rects, const uint32_t* offsets,
                        long long R, uint64_t* keys, uint32_t* vals, int32_t* owner_count)
{
    int gw = (cfg->W + 15) / 16, gh = (cfg->H + 15) / 16;
    long long prev_reach = 0, dropped = 0;
    for (int i = 0; i < P; ++i) {
        if (radii[i] <= 0) continue;
        long long start = i == 0 ? 0 : (long long)offsets[i - 1];
        int x0, y0, x1, y1;
        if (cfg->compat_spill) {
            REAL cx = means2D[2 * i], cy = means2D[2 * i + 1];
            REAL rad = (REAL)radii[i];
            int a = (int)RFLOOR((cx - rad) / (REAL)16), b = (int)RCEIL((cx + rad) / (REAL)16);
            int c = (int)RFLOOR((cy - rad) / (REAL)16), d = (int)RCEIL((cy + rad) / (REAL)16);
            x0 = a < 0 ? 0 : (a > gw ? gw : a); x1 = b < 0 ? 0 : (b > gw ? gw : b);
            y0 = c < 0 ? 0 : (c > gh ? gh : c); y1 = d < 0 ? 0 : (d > gh ? gh : d);
        } else {
            x0 = rects[4 * i]; y0 = rects[4 * i + 1]; x1 = rects[4 * i + 2]; y1 = rects[4 * i + 3];
        }
        int w = x1 - x0, h = y1 - y0;
        long long n = (w > 0 && h > 0) ? (long long)w * h : 0;
        long long reach = start + n;
        long long p0 = start > prev_reach ? start : prev_reach;
        uint32_t dbits;
        float df = (float)depth[i];
        memcpy(&dbits, &df, 4);
        for (long long p = start; p < reach; ++p) {
            if (p >= R) { if (p >= p0) dropped++; continue; }
            if (owner_count) owner_count[p]++; /* candidate writers of slot p */
            if (p < p0) continue;               /* a lower index already owns p */
            long long k = p - start;
            int tx = x0 + (int)(k % w), ty = y0 + (int)(k / w);
            uint32_t tile = (uint32_t)(ty * gw + tx);
            keys[p] = ((uint64_t)tile << 32) | dbits;
            vals[p] = (uint32_t)i;
        }
        if (reach > prev_reach) prev_reach = reach;
    }
    return dropped;
}

/* ------------------------------------------------------------------------ */
/* Forward: per-tile alpha blending                                          */
/* (pixelGaussiansFull.cu:57-97, pixelGaussiansDev.cuh:20-84, gaussEval.h:13-28) */
/* ------------------------------------------------------------------------ */
/* Gaussian value at a pixel from the 2-D covariance and its determinant,
 * gaussEval.h:13-28 (mahalanobis / det, negative -> 1000). */
static inline REAL SFX(gauss_eval)(REAL mux, REAL muy, REAL cxx, REAL cxy, REAL cyy, REAL det,
                                   REAL qx, REAL qy)
{
    REAL dx = qx - mux, dy = qy - muy;
    REAL tX = SFX(d2)(orc_var[V_BL_TX], dx, cyy, dy, cxy);
    REAL tY = SFX(s2)(orc_var[V_BL_TY], -dx, cxy, dy, cxx);
    REAL num = SFX(s2)(orc_var[V_BL_NUM], tX, dx, tY, dy);
    REAL m = num / det;
    if (m < (REAL)0) m = (REAL)1000;
    return REXP((REAL)-0.5 * m);
}

/* The blend's own determinant of the 2-D covariance (gaussEval.h:21). */
static inline REAL SFX(blend_det)(const REAL* cov2D) {
    return SFX(d2)(orc_var[V_BL_DET], cov2D[0], cov2D[2], cov2D[1], cov2D[1]);
}

/* ranges: T x 2 (start, end) per tile; point_list: Gaussian ids in sorted
 * order.  Outputs: color[3*H*W] (CHW), depth[H*W], alpha[H*W] (= sum of
 * alpha*T, pixelGaussiansFull.cu:355), n_contrib[H*W] (1-based index of the
 * last blended entry of the tile's list).  bg is added with the final
 * transmittance (the reference hard-codes white, :360); out_T[H*W] (may be
 * NULL) receives the final transmittance.  margin[H*W] (may be
 * NULL): smallest relative distance of any alpha or transmittance test of the
 * pixel from its threshold.  sig[H*W] (may be NULL): a hash of the pixel's
 * blend decisions (which entries were blended, which hit the 0.99 clamp),
 * so callers can tell when a perturbation changed a discrete decision. */
typedef struct {
    const orc_cfg* cfg;
    const uint32_t* ranges;
    const uint32_t* point_list;
    const REAL* means2D;
    const REAL* cov2D;
    const REAL* conic_opac;
    const REAL* rgb;
    const REAL* depth;
    REAL* out_color;
    REAL* out_depth;
    REAL* out_alpha;
    uint32_t* n_contrib;
    REAL* out_T;
    double* margin;
    uint64_t* sig;
} SFX(orc_blend_ctx);
static void SFX(orc_blend_part)(void* vc_, long long lo_, long long hi_, int tid_)
{
    SFX(orc_blend_ctx)* c_ = (SFX(orc_blend_ctx)*)vc_;
    const orc_cfg* cfg = c_->cfg;
    const uint32_t* ranges = c_->ranges;
    const uint32_t* point_list = c_->point_list;
    const REAL* means2D = c_->means2D;
    const REAL* cov2D = c_->cov2D;
    const REAL* conic_opac = c_->conic_opac;
    const REAL* rgb = c_->rgb;
    const REAL* depth = c_->depth;
    REAL* out_color = c_->out_color;
    REAL* out_depth = c_->out_depth;
    REAL* out_alpha = c_->out_alpha;
    uint32_t* n_contrib = c_->n_contrib;
    REAL* out_T = c_->out_T;
    double* margin = c_->margin;
    uint64_t* sig = c_->sig;
    (void)tid_;

    const int W = cfg->W, H = cfg->H, gw = (W + 15) / 16;
    const REAL min_alpha = (REAL)(1.0f / 255.0f), min_T = (REAL)0.0001f, max_alpha = (REAL)0.99f;
    for (int py = (int)lo_; py < (int)hi_; ++py) {
        for (int px = 0; px < W; ++px) {
            int tile = (py / 16) * gw + (px / 16);
            uint32_t s = ranges[2 * tile], e = ranges[2 * tile + 1];
            REAL C[3] = {0, 0, 0}, Wt = 0, D = 0, T = 1;
            uint32_t contributor = 0, last = 0;
            double mg = 1e30;
            uint64_t hs = 1469598103934665603ull;
            REAL qx = (REAL)px, qy = (REAL)py;
            for (uint32_t j = s; j < e; ++j) {
                uint32_t id = point_list[j];
                ++contributor;
                REAL det = SFX(blend_det)(cov2D + 3 * id);
                REAL g = SFX(gauss_eval)(means2D[2 * id], means2D[2 * id + 1], cov2D[3 * id],
                                         cov2D[3 * id + 1], cov2D[3 * id + 2], det, qx, qy);
                REAL o = conic_opac[4 * id + 3];
                REAL og = o * g;
                REAL a = og < max_alpha ? og : max_alpha;
                double ma = fabs((double)a - (double)min_alpha) / (double)min_alpha;
                if (ma < mg) mg = ma;
                if (a >= min_alpha) {
                    REAL nT = T * ((REAL)1 - a);
                    double mt = fabs((double)nT - (double)min_T) / (double)min_T;
                    if (mt < mg) mg = mt;
                    if (nT >= min_T) {
                        REAL aT = a * T;
                        for (int c = 0; c < 3; ++c) C[c] = RFMA(rgb[3 * id + c], aT, C[c]);
                        Wt = Wt + aT;
                        D = SFX(s1)(orc_var[V_BL_DEPTH], depth[id], aT, D);
                        T = nT;
                        last = contributor;
                        hs = (hs ^ (uint64_t)(2u * contributor + (og < max_alpha ? 0u : 1u))) * 1099511628211ull;
                    } else {
                        break;
                    }
                }
            }
            size_t pix = (size_t)py * W + px;
            n_contrib[pix] = last;
            out_alpha[pix] = Wt;
            out_depth[pix] = D;
            for (int c = 0; c < 3; ++c)
                out_color[(size_t)c * H * W + pix] = RFMA(T, (REAL)cfg->bg[c], C[c]);
            if (margin) margin[pix] = mg;
            if (out_T) out_T[pix] = T;
            if (sig) sig[pix] = hs;
        }
    }
}

void SFX(orc_blend)(const orc_cfg* cfg, const uint32_t* ranges, const uint32_t* point_list,
                    const REAL* means2D, const REAL* cov2D, const REAL* conic_opac,
                    const REAL* rgb, const REAL* depth,
                    REAL* out_color, REAL* out_depth, REAL* out_alpha, uint32_t* n_contrib,
                    REAL* out_T, double* margin, uint64_t* sig)
{
    SFX(orc_blend_ctx) c_ = {cfg, ranges, point_list, means2D, cov2D, conic_opac, rgb, depth, out_color, out_depth, out_alpha, n_contrib, out_T, margin, sig};
    orc_parallel_for(cfg->H, 1, SFX(orc_blend_part), &c_);
}


/* ------------------------------------------------------------------------ */
/* Backward: per-pixel gradients, back to front (backward.cu:521-665)       */
/* ------------------------------------------------------------------------ */
/* Reference-gradient mode.  Accumulates in double (the reference uses float
 * atomics in an unspecified order).  Outputs (zeroed by the caller):
 *   dmean2D[P*3] (x, y used), dconic[P*4] (x, y, w used), dopac[P],
 *   dcolor[P*3], ddepth[P].
 * The pixel-to-NDC factors 0.5*W and 0.5*H come from the gradient image size
 * (backward.cu:586-587). */
typedef struct {
    const orc_cfg* cfg; int P; const uint32_t* ranges; const uint32_t* point_list;
    const REAL* means2D; const REAL* conic_opac; const REAL* rgb; const REAL* depth; const REAL* out_alpha;
    const uint32_t* n_contrib; const float* dL_dpix; const float* dL_ddepth; const float* dL_dalpha;
    double* dmean2D; double* dconic; double* dopac; double* dcolor; double* ddepth; double* abs_sum;
    double* priv; size_t stride; double* margin;
} SFX(orc_backward_render_ctx);

/* Rows [lo_, hi_) of the per-pixel backward.  With several threads each
 * accumulates into its own zeroed copy of the outputs (priv), summed in
 * thread order at the end. */
static void SFX(orc_backward_render_part)(void* vc_, long long lo_, long long hi_, int tid_)
{
    SFX(orc_backward_render_ctx)* c_ = (SFX(orc_backward_render_ctx)*)vc_;
    const orc_cfg* cfg = c_->cfg; const uint32_t* ranges = c_->ranges; const uint32_t* point_list = c_->point_list;
    const REAL* means2D = c_->means2D; const REAL* conic_opac = c_->conic_opac; const REAL* rgb = c_->rgb;
    const REAL* depth = c_->depth; const REAL* out_alpha = c_->out_alpha; const uint32_t* n_contrib = c_->n_contrib;
    const float* dL_dpix = c_->dL_dpix; const float* dL_ddepth = c_->dL_ddepth; const float* dL_dalpha = c_->dL_dalpha;
    double *m2 = c_->dmean2D, *cn = c_->dconic, *op = c_->dopac, *cl = c_->dcolor, *dp = c_->ddepth, *as_ = c_->abs_sum;
    if (c_->priv) {
        const size_t P = (size_t)c_->P;
        double* b = c_->priv + (size_t)tid_ * P * c_->stride;
        m2 = b; cn = b + 3 * P; op = b + 7 * P; cl = b + 8 * P; dp = b + 11 * P;
        as_ = c_->abs_sum ? b + 12 * P : NULL;
    }

    /* abs_sum[P*10] (may be NULL): per Gaussian, the sum of |contribution| of
     * each accumulated value (colour r,g,b, depth, mean2D x,y, conic x,y,w,
     * opacity) -- the scale of fp32 accumulation-order error */
    const int W = cfg->W, H = cfg->H, gw = (W + 15) / 16;
    const REAL ddelx_dx = (REAL)(0.5 * W), ddely_dy = (REAL)(0.5 * H);
    const REAL bg[3] = {cfg->bg[0], cfg->bg[1], cfg->bg[2]};
    for (int py = (int)lo_; py < (int)hi_; ++py) {
        for (int px = 0; px < W; ++px) {
            int tile = (py / 16) * gw + (px / 16);
            uint32_t s = ranges[2 * tile], e = ranges[2 * tile + 1];
            size_t pix = (size_t)py * W + px;
            const REAL Tf = (REAL)1 - out_alpha[pix];
            REAL T = Tf;
            uint32_t contributor = e - s;
            uint32_t last = n_contrib[pix];
            REAL dLp[3];
            for (int c = 0; c < 3; ++c) dLp[c] = dL_dpix[(size_t)c * H * W + pix];
            REAL dLd = dL_ddepth[pix], dLa = dL_dalpha[pix];
            REAL acc[3] = {0, 0, 0}, accd = 0, acca = 0, last_a = 0, last_c[3] = {0, 0, 0}, last_d = 0;
            REAL bgdot = 0;
            for (int c = 0; c < 3; ++c) bgdot = bgdot + bg[c] * dLp[c];
            REAL qx = (REAL)px, qy = (REAL)py;
            double mg = 1e30;  /* smallest relative distance of a skip decision from its threshold */
            for (uint32_t jj = e; jj > s; --jj) {
                uint32_t j = jj - 1;
                contributor--;
                if (contributor >= last) continue;
                uint32_t id = point_list[j];
                REAL dx = means2D[2 * id] - qx, dy = means2D[2 * id + 1] - qy;
                const REAL* co = conic_opac + 4 * id;
                REAL power = (REAL)-0.5 * (co[0] * dx * dx + co[2] * dy * dy) - co[1] * dx * dy;
                if (fabs((double)power) < 1e-6 && mg > 0) mg = 0; /* at the power > 0 test */
                if (power > (REAL)0) continue;
                REAL G = REXP(power);
                REAL og = co[3] * G;
                REAL a = og < (REAL)0.99f ? og : (REAL)0.99f;
                {
                    const double ma = fabs((double)a - 1.0 / 255.0) * 255.0;
                    if (ma < mg) mg = ma;
                }
                if (a < (REAL)(1.0f / 255.0f)) continue;
                T = T / ((REAL)1 - a);
                REAL dchdc = a * T;
                REAL dLdo = 0;
                for (int c = 0; c < 3; ++c) {
                    REAL col = rgb[3 * id + c];
                    acc[c] = last_a * last_c[c] + ((REAL)1 - last_a) * acc[c];
                    last_c[c] = col;
                    dLdo = dLdo + (col - acc[c]) * dLp[c];
                    cl[3 * id + c] += (double)(dchdc * dLp[c]);
                }
                REAL cd = depth[id];
                accd = last_a * last_d + ((REAL)1 - last_a) * accd;
                last_d = cd;
                dLdo = dLdo + (cd - accd) * dLd;
                dp[id] += (double)(a * T * dLd);
                acca = last_a + ((REAL)1 - last_a) * acca;
                dLdo = dLdo + ((REAL)1 - acca) * dLa;
                dLdo = dLdo * T;
                last_a = a;
                dLdo = dLdo + (-Tf / ((REAL)1 - a)) * bgdot;
                REAL dLdG = co[3] * dLdo;
                REAL gdx = G * dx, gdy = G * dy;
                REAL dGdx = -gdx * co[0] - gdy * co[1];
                REAL dGdy = -gdy * co[2] - gdx * co[1];
                m2[3 * id] += (double)(dLdG * dGdx * ddelx_dx);
                m2[3 * id + 1] += (double)(dLdG * dGdy * ddely_dy);
                cn[4 * id] += (double)((REAL)-0.5 * gdx * dx * dLdG);
                cn[4 * id + 1] += (double)((REAL)-0.5 * gdx * dy * dLdG);
                cn[4 * id + 3] += (double)((REAL)-0.5 * gdy * dy * dLdG);
                op[id] += (double)(G * dLdo);
                if (as_) {
                    double* as = as_ + 10 * (size_t)id;
                    for (int c = 0; c < 3; ++c) as[c] += fabs((double)(dchdc * dLp[c]));
                    as[3] += fabs((double)(a * T * dLd));
                    as[4] += fabs((double)(dLdG * dGdx * ddelx_dx));
                    as[5] += fabs((double)(dLdG * dGdy * ddely_dy));
                    as[6] += fabs((double)((REAL)-0.5 * gdx * dx * dLdG));
                    as[7] += fabs((double)((REAL)-0.5 * gdx * dy * dLdG));
                    as[8] += fabs((double)((REAL)-0.5 * gdy * dy * dLdG));
                    as[9] += fabs((double)(G * dLdo));
                }
            }
            if (c_->margin) c_->margin[pix] = mg;
        }
    }
}

void SFX(orc_backward_render)(const orc_cfg* cfg, int P, const uint32_t* ranges, const uint32_t* point_list,
                              const REAL* means2D, const REAL* conic_opac, const REAL* rgb,
                              const REAL* depth, const REAL* out_alpha, const uint32_t* n_contrib,
                              const float* dL_dpix, const float* dL_ddepth, const float* dL_dalpha,
                              double* dmean2D, double* dconic, double* dopac, double* dcolor,
                              double* ddepth, double* abs_sum, double* margin)
{
    /* margin[H*W] (may be NULL): per pixel, the smallest relative distance of
     * a walked pair's recomputed alpha from the 1/255 skip threshold (0 where
     * the exponent is within 1e-6 of the power > 0 test): the device's exp
     * and the C library's may decide such a pair differently */
    /* abs_sum[P*10] (may be NULL): per Gaussian, the sum of |contribution| of
     * each accumulated value (colour r,g,b, depth, mean2D x,y, conic x,y,w,
     * opacity) -- the scale of fp32 accumulation-order error */
    const int nt = orc_threads > 1 ? orc_threads : 1;
    const size_t stride = abs_sum ? 22 : 12;
    double* priv = nt > 1 ? (double*)calloc((size_t)nt * (size_t)P * stride, sizeof(double)) : NULL;
    SFX(orc_backward_render_ctx) c_ = {cfg, P, ranges, point_list, means2D, conic_opac, rgb, depth, out_alpha,
                                       n_contrib, dL_dpix, dL_ddepth, dL_dalpha, dmean2D, dconic, dopac, dcolor,
                                       ddepth, abs_sum, priv, stride, margin};
    if (priv == NULL) {
        SFX(orc_backward_render_part)(&c_, 0, cfg->H, 0);
        return;
    }
    orc_parallel_for(cfg->H, 1, SFX(orc_backward_render_part), &c_);
    for (int t = 0; t < nt; ++t) {
        const double* b = priv + (size_t)t * (size_t)P * stride;
        const size_t Pz = (size_t)P;
        for (size_t i = 0; i < 3 * Pz; ++i) dmean2D[i] += b[i];
        for (size_t i = 0; i < 4 * Pz; ++i) dconic[i] += b[3 * Pz + i];
        for (size_t i = 0; i < Pz; ++i) dopac[i] += b[7 * Pz + i];
        for (size_t i = 0; i < 3 * Pz; ++i) dcolor[i] += b[8 * Pz + i];
        for (size_t i = 0; i < Pz; ++i) ddepth[i] += b[11 * Pz + i];
        if (abs_sum)
            for (size_t i = 0; i < 10 * Pz; ++i) abs_sum[i] += b[12 * Pz + i];
    }
    free(priv);
}

/* ------------------------------------------------------------------------ */
/* Backward: dL/dconic -> dL/dcov3D and the Jacobian part of dL/dmean3D     */
/* (backward.cu:27-227)                                                     */
/* ------------------------------------------------------------------------ */
/* h_x, h_y = W/(2 tan_fovx), H/(2 tan_fovy) (gradientPass.cu:119-120).
 * ASSIGNS dmean3D for visible Gaussians (backward.cu:226). */
typedef struct {
    int P;
    const float* means3D;
    const int32_t* radii;
    const REAL* cov3D;
    REAL h_x;
    REAL h_y;
    REAL tan_fovx;
    REAL tan_fovy;
    const float* view;
    const REAL* dconic;
    REAL* dcov3D;
    REAL* dmean3D;
} SFX(orc_backward_cov2d_ctx);
static void SFX(orc_backward_cov2d_part)(void* vc_, long long lo_, long long hi_, int tid_)
{
    SFX(orc_backward_cov2d_ctx)* c_ = (SFX(orc_backward_cov2d_ctx)*)vc_;
    (void)c_->P;
    const float* means3D = c_->means3D;
    const int32_t* radii = c_->radii;
    const REAL* cov3D = c_->cov3D;
    REAL h_x = c_->h_x;
    REAL h_y = c_->h_y;
    REAL tan_fovx = c_->tan_fovx;
    REAL tan_fovy = c_->tan_fovy;
    const float* view = c_->view;
    const REAL* dconic = c_->dconic;
    REAL* dcov3D = c_->dcov3D;
    REAL* dmean3D = c_->dmean3D;
    (void)tid_;

    for (int i = (int)lo_; i < (int)hi_; ++i) {
        if (!(radii[i] > 0)) continue;
        const REAL* pc = cov3D + 6 * i;
        REAL cx = means3D[3 * i], cy = means3D[3 * i + 1], cz = means3D[3 * i + 2];
        REAL vx = view[0] * cx + view[4] * cy + view[8] * cz + view[12];
        REAL vy = view[1] * cx + view[5] * cy + view[9] * cz + view[13];
        REAL vz = view[2] * cx + view[6] * cy + view[10] * cz + view[14];
        REAL vw = view[3] * cx + view[7] * cy + view[11] * cz + view[15];
        REAL winv = (REAL)1 / (vw + (REAL)1e-8f);
        vx *= winv; vy *= winv; vz *= winv;
        REAL bx = (REAL)1.3f * tan_fovx, by = (REAL)1.3f * tan_fovy;
        REAL prx = vx / vz, pry = vy / vz;
        REAL cpx = prx < -bx ? -bx : prx; cpx = cpx > bx ? bx : cpx;
        REAL cpy = pry < -by ? -by : pry; cpy = cpy > by ? by : cpy;
        REAL px = cpx * vz, py = cpy * vz;
        REAL mxk = (prx >= -bx && prx <= bx) ? (REAL)1 : (REAL)0;
        REAL myk = (pry >= -by && pry <= by) ? (REAL)1 : (REAL)0;
        REAL zi = (REAL)1 / vz, zi2 = zi * zi;
        /* glm column-major: J[col][row] */
        REAL J[3][3] = {{h_x * zi, 0, -h_x * px * zi2}, {0, h_y * zi, -h_y * py * zi2}, {0, 0, 0}};
        REAL Wv[3][3] = {{view[0], view[4], view[8]}, {view[1], view[5], view[9]}, {view[2], view[6], view[10]}};
        REAL Vk[3][3] = {{pc[0], pc[1], pc[2]}, {pc[1], pc[3], pc[4]}, {pc[2], pc[4], pc[5]}};
        REAL T[3][3], tmp[3][3], c2[3][3];
        /* T = Wv * J (glm product: Result[c][r] = sum_k A[k][r] * B[c][k]) */
        for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r)
            T[c][r] = Wv[0][r] * J[c][0] + Wv[1][r] * J[c][1] + Wv[2][r] * J[c][2];
        /* temp = transpose(Vk) * T ; cov2 = transpose(T) * temp */
        REAL VkT[3][3], TT[3][3];
        for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r) { VkT[c][r] = Vk[r][c]; TT[c][r] = T[r][c]; }
        for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r)
            tmp[c][r] = VkT[0][r] * T[c][0] + VkT[1][r] * T[c][1] + VkT[2][r] * T[c][2];
        for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r)
            c2[c][r] = TT[0][r] * tmp[c][0] + TT[1][r] * tmp[c][1] + TT[2][r] * tmp[c][2];
        c2[0][0] += (REAL)0.3f;
        c2[1][1] += (REAL)0.3f;
        REAL a = c2[0][0], b = c2[0][1], c = c2[1][1];
        REAL den = a * c - b * b;
        REAL dinv2 = (REAL)1 / (den * den + (REAL)1e-7f);
        REAL gx = dconic[4 * i], gy = dconic[4 * i + 1], gz = dconic[4 * i + 3];
        REAL ga = 0, gb = 0, gc = 0;
        REAL* dc = dcov3D + 6 * i;
        if (dinv2 > (REAL)0) {
            ga = dinv2 * (-c * c * gx + (REAL)2 * b * c * gy + (den - a * c) * gz);
            gb = dinv2 * (REAL)2 * (b * c * gx - (den + (REAL)2 * b * b) * gy + a * b * gz);
            gc = dinv2 * (-a * a * gz + (REAL)2 * a * b * gy + (den - a * c) * gx);
            dc[0] = T[0][0] * T[0][0] * ga + T[0][0] * T[1][0] * gb + T[1][0] * T[1][0] * gc;
            dc[3] = T[0][1] * T[0][1] * ga + T[0][1] * T[1][1] * gb + T[1][1] * T[1][1] * gc;
            dc[5] = T[0][2] * T[0][2] * ga + T[0][2] * T[1][2] * gb + T[1][2] * T[1][2] * gc;
            dc[1] = (REAL)2 * (T[0][0] * T[0][1] * ga + (T[0][0] * T[1][1] + T[0][1] * T[1][0]) * gb * (REAL)0.5 + T[1][0] * T[1][1] * gc);
            dc[2] = (REAL)2 * (T[0][0] * T[0][2] * ga + (T[0][0] * T[1][2] + T[0][2] * T[1][0]) * gb * (REAL)0.5 + T[1][0] * T[1][2] * gc);
            dc[4] = (REAL)2 * (T[0][1] * T[0][2] * ga + (T[0][1] * T[1][2] + T[0][2] * T[1][1]) * gb * (REAL)0.5 + T[1][1] * T[1][2] * gc);
        } else {
            for (int k = 0; k < 6; ++k) dc[k] = 0;
        }
        REAL gT00 = (REAL)2 * (T[0][0] * Vk[0][0] + T[0][1] * Vk[0][1] + T[0][2] * Vk[0][2]) * ga + (T[1][0] * Vk[0][0] + T[1][1] * Vk[0][1] + T[1][2] * Vk[0][2]) * gb;
        REAL gT01 = (REAL)2 * (T[0][0] * Vk[1][0] + T[0][1] * Vk[1][1] + T[0][2] * Vk[1][2]) * ga + (T[1][0] * Vk[1][0] + T[1][1] * Vk[1][1] + T[1][2] * Vk[1][2]) * gb;
        REAL gT02 = (REAL)2 * (T[0][0] * Vk[2][0] + T[0][1] * Vk[2][1] + T[0][2] * Vk[2][2]) * ga + (T[1][0] * Vk[2][0] + T[1][1] * Vk[2][1] + T[1][2] * Vk[2][2]) * gb;
        REAL gT10 = (REAL)2 * (T[1][0] * Vk[0][0] + T[1][1] * Vk[0][1] + T[1][2] * Vk[0][2]) * gc + (T[0][0] * Vk[0][0] + T[0][1] * Vk[0][1] + T[0][2] * Vk[0][2]) * gb;
        REAL gT11 = (REAL)2 * (T[1][0] * Vk[1][0] + T[1][1] * Vk[1][1] + T[1][2] * Vk[1][2]) * gc + (T[0][0] * Vk[1][0] + T[0][1] * Vk[1][1] + T[0][2] * Vk[1][2]) * gb;
        REAL gT12 = (REAL)2 * (T[1][0] * Vk[2][0] + T[1][1] * Vk[2][1] + T[1][2] * Vk[2][2]) * gc + (T[0][0] * Vk[2][0] + T[0][1] * Vk[2][1] + T[0][2] * Vk[2][2]) * gb;
        REAL gJ00 = Wv[0][0] * gT00 + Wv[0][1] * gT01 + Wv[0][2] * gT02;
        REAL gJ02 = Wv[2][0] * gT00 + Wv[2][1] * gT01 + Wv[2][2] * gT02;
        REAL gJ11 = Wv[1][0] * gT10 + Wv[1][1] * gT11 + Wv[1][2] * gT12;
        REAL gJ12 = Wv[2][0] * gT10 + Wv[2][1] * gT11 + Wv[2][2] * gT12;
        REAL zi3 = zi2 * zi;
        REAL gvx = mxk * (-h_x * zi2 * gJ02);
        REAL gvy = myk * (-h_y * zi2 * gJ12);
        REAL gvz = -h_x * zi2 * gJ00 - h_y * zi2 * gJ11 + (REAL)2 * h_x * px * zi3 * gJ02 + (REAL)2 * h_y * py * zi3 * gJ12;
        dmean3D[3 * i] = view[0] * gvx + view[1] * gvy + view[2] * gvz;
        dmean3D[3 * i + 1] = view[4] * gvx + view[5] * gvy + view[6] * gvz;
        dmean3D[3 * i + 2] = view[8] * gvx + view[9] * gvy + view[10] * gvz;
    }
}

void SFX(orc_backward_cov2d)(int P, const float* means3D, const int32_t* radii, const REAL* cov3D,
                             REAL h_x, REAL h_y, REAL tan_fovx, REAL tan_fovy, const float* view,
                             const REAL* dconic, REAL* dcov3D, REAL* dmean3D)
{
    SFX(orc_backward_cov2d_ctx) c_ = {P, means3D, radii, cov3D, h_x, h_y, tan_fovx, tan_fovy, view, dconic, dcov3D, dmean3D};
    orc_parallel_for(P, 4096, SFX(orc_backward_cov2d_part), &c_);
}


/* ------------------------------------------------------------------------ */
/* Backward: mean2D/depth -> mean3D, SH, scale and rotation gradients       */
/* (backward.cu:229-519)                                                    */
/* ------------------------------------------------------------------------ */
typedef struct {
    int P;
    int M;
    const float* means3D;
    const int32_t* radii;
    const float* sh;
    const uint8_t* clamped;
    const float* scales;
    const float* rots;
    REAL scale_mod;
    const float* view;
    const float* proj;
    const float* campos;
    const REAL* dmean2D;
    const REAL* dcolor;
    const REAL* ddepth;
    const REAL* dcov3D;
    REAL* dmean3D;
    REAL* dsh;
    REAL* dscale;
    REAL* drot;
} SFX(orc_backward_preprocess_ctx);
static void SFX(orc_backward_preprocess_part)(void* vc_, long long lo_, long long hi_, int tid_)
{
    SFX(orc_backward_preprocess_ctx)* c_ = (SFX(orc_backward_preprocess_ctx)*)vc_;
    (void)c_->P;
    int M = c_->M;
    const float* means3D = c_->means3D;
    const int32_t* radii = c_->radii;
    const float* sh = c_->sh;
    const uint8_t* clamped = c_->clamped;
    const float* scales = c_->scales;
    const float* rots = c_->rots;
    REAL scale_mod = c_->scale_mod;
    const float* view = c_->view;
    const float* proj = c_->proj;
    const float* campos = c_->campos;
    const REAL* dmean2D = c_->dmean2D;
    const REAL* dcolor = c_->dcolor;
    const REAL* ddepth = c_->ddepth;
    const REAL* dcov3D = c_->dcov3D;
    REAL* dmean3D = c_->dmean3D;
    REAL* dsh = c_->dsh;
    REAL* dscale = c_->dscale;
    REAL* drot = c_->drot;
    (void)tid_;

    static const REAL C0 = (REAL)0.28209479177387814f, C1 = (REAL)0.4886025119029199f;
    static const REAL C2[5] = {(REAL)1.0925484305920792f, (REAL)-1.0925484305920792f, (REAL)0.31539156525252005f,
                               (REAL)-1.0925484305920792f, (REAL)0.5462742152960396f};
    static const REAL C3[7] = {(REAL)-0.5900435899266435f, (REAL)2.890611442640554f, (REAL)-0.4570457994644658f,
                               (REAL)0.3731763325901154f, (REAL)-0.4570457994644658f, (REAL)1.445305721320277f,
                               (REAL)-0.5900435899266435f};
    for (int i = (int)lo_; i < (int)hi_; ++i) {
        if (radii[i] <= 0) continue;
        REAL wx = means3D[3 * i], wy = means3D[3 * i + 1], wz = means3D[3 * i + 2];
        const float* m = proj;
        REAL cw = m[3] * wx + m[7] * wy + m[11] * wz + m[15];
        REAL iw = (REAL)1 / (cw + (REAL)1e-7f);
        REAL iw2 = iw * iw;
        REAL ptx = (m[0] * wx + m[4] * wy + m[8] * wz + m[12]) * iw2;
        REAL pty = (m[1] * wx + m[5] * wy + m[9] * wz + m[13]) * iw2;
        REAL g2x = dmean2D[3 * i], g2y = dmean2D[3 * i + 1];
        REAL sd[3] = {dmean3D[3 * i], dmean3D[3 * i + 1], dmean3D[3 * i + 2]};
        sd[0] += (m[0] * iw - m[3] * ptx) * g2x + (m[1] * iw - m[3] * pty) * g2y;
        sd[1] += (m[4] * iw - m[7] * ptx) * g2x + (m[5] * iw - m[7] * pty) * g2y;
        sd[2] += (m[8] * iw - m[11] * ptx) * g2x + (m[9] * iw - m[11] * pty) * g2y;
        REAL vz = view[2] * wx + view[6] * wy + view[10] * wz + view[14];
        REAL gd = ddepth[i];
        sd[0] += (view[2] - view[3] * vz) * gd;
        sd[1] += (view[6] - view[7] * vz) * gd;
        sd[2] += (view[10] - view[11] * vz) * gd;
        /* SH (backward.cu:291-444): all 16 bands regardless of degree */
        REAL ox = wx - campos[0], oy = wy - campos[1], oz = wz - campos[2];
        REAL msq = ox * ox + oy * oy + oz * oz;
        REAL mag = RSQRT(msq + (REAL)1e-10f);
        REAL im = (REAL)1 / mag;
        REAL x = ox * im, y = oy * im, z = oz * im;
        REAL x2 = x * x, y2 = y * y, z2 = z * z, xy = x * y, xz = x * z, yz = y * z;
        REAL x2my2 = x2 - y2, tx2 = (REAL)3 * x2, ty2 = (REAL)3 * y2, fz2 = (REAL)4 * z2, wz2 = (REAL)2 * z2;
        REAL cf[3];
        for (int c = 0; c < 3; ++c) cf[c] = dcolor[3 * i + c] * (clamped[3 * i + c] ? (REAL)0 : (REAL)1);
        const float* sdat = sh + (size_t)i * M * 3;
        REAL basis[16];
        basis[0] = C0; basis[1] = -C1 * y; basis[2] = C1 * z; basis[3] = -C1 * x;
        basis[4] = C2[0] * xy; basis[5] = C2[1] * yz; basis[6] = C2[2] * (wz2 - x2 - y2);
        basis[7] = C2[3] * xz; basis[8] = C2[4] * x2my2;
        basis[9] = C3[0] * y * (tx2 - y2); basis[10] = C3[1] * xy * z; basis[11] = C3[2] * y * (fz2 - x2 - y2);
        basis[12] = C3[3] * z * (wz2 - tx2 - ty2); basis[13] = C3[4] * x * (fz2 - x2 - y2);
        basis[14] = C3[5] * z * x2my2; basis[15] = C3[6] * x * (x2 - ty2);
        int nb = M < 16 ? M : 16;
        for (int k = 0; k < nb; ++k)
            for (int c = 0; c < 3; ++c) dsh[((size_t)i * M + k) * 3 + c] = basis[k] * cf[c];
        REAL ag[3] = {0, 0, 0};
#define SHV(k, c) ((REAL)((k) < M ? sdat[3 * (k) + (c)] : 0.0f))
#define DOTC(k) (SHV(k, 0) * cf[0] + SHV(k, 1) * cf[1] + SHV(k, 2) * cf[2])
        ag[0] -= C1 * DOTC(3);
        ag[1] -= C1 * DOTC(1);
        ag[2] += C1 * DOTC(2);
        REAL d2x[3], d2y[3], d2z[3];
        for (int c = 0; c < 3; ++c) {
            d2x[c] = C2[0] * y * SHV(4, c) + C2[2] * ((REAL)-2 * x) * SHV(6, c) + C2[3] * z * SHV(7, c) + C2[4] * ((REAL)2 * x) * SHV(8, c);
            d2y[c] = C2[0] * x * SHV(4, c) + C2[1] * z * SHV(5, c) + C2[2] * ((REAL)-2 * y) * SHV(6, c) + C2[4] * ((REAL)-2 * y) * SHV(8, c);
            d2z[c] = C2[1] * y * SHV(5, c) + C2[2] * ((REAL)4 * z) * SHV(6, c) + C2[3] * x * SHV(7, c);
        }
        ag[0] += d2x[0] * cf[0] + d2x[1] * cf[1] + d2x[2] * cf[2];
        ag[1] += d2y[0] * cf[0] + d2y[1] * cf[1] + d2y[2] * cf[2];
        ag[2] += d2z[0] * cf[0] + d2z[1] * cf[1] + d2z[2] * cf[2];
        REAL f3x[7] = {C3[0] * (REAL)6 * xy, C3[1] * yz, C3[2] * ((REAL)-2 * xy), C3[3] * ((REAL)-6 * xz),
                       C3[4] * (fz2 - (REAL)3 * x2 - y2), C3[5] * (REAL)2 * xz, C3[6] * (REAL)3 * x2my2};
        REAL f3y[7] = {C3[0] * (REAL)3 * (x2 - y2), C3[1] * xz, C3[2] * (fz2 - (REAL)3 * y2 - x2), C3[3] * ((REAL)-6 * yz),
                       C3[4] * ((REAL)-2 * xy), C3[5] * ((REAL)-2 * yz), C3[6] * ((REAL)-6 * xy)};
        REAL f3z[7] = {0, C3[1] * xy, C3[2] * (REAL)8 * yz, C3[3] * (REAL)3 * (wz2 - x2 - y2),
                       C3[4] * (REAL)8 * xz, C3[5] * x2my2, 0};
        REAL d3x[3] = {0, 0, 0}, d3y[3] = {0, 0, 0}, d3z[3] = {0, 0, 0};
        for (int k = 0; k < 7; ++k)
            for (int c = 0; c < 3; ++c) {
                d3x[c] += f3x[k] * SHV(9 + k, c);
                d3y[c] += f3y[k] * SHV(9 + k, c);
                d3z[c] += f3z[k] * SHV(9 + k, c);
            }
        ag[0] += d3x[0] * cf[0] + d3x[1] * cf[1] + d3x[2] * cf[2];
        ag[1] += d3y[0] * cf[0] + d3y[1] * cf[1] + d3y[2] * cf[2];
        ag[2] += d3z[0] * cf[0] + d3z[1] * cf[1] + d3z[2] * cf[2];
#undef DOTC
#undef SHV
        REAL im3 = im * im * im;
        REAL rd[3] = {ox, oy, oz};
        REAL jac[3][3];
        for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r)
            jac[c][r] = ((c == r ? msq : (REAL)0) - rd[c] * rd[r]) * im3;
        for (int r = 0; r < 3; ++r)
            sd[r] += jac[0][r] * ag[0] + jac[1][r] * ag[1] + jac[2][r] * ag[2];
        dmean3D[3 * i] = sd[0]; dmean3D[3 * i + 1] = sd[1]; dmean3D[3 * i + 2] = sd[2];

        /* scale / rotation (backward.cu:446-518) */
        const float* q = rots + 4 * i;
        REAL qw = q[0], qx = q[1], qy = q[2], qz = q[3];
        REAL xx = qx * qx, yy = qy * qy, zz = qz * qz;
        REAL qxy = qx * qy, qxz = qx * qz, qyz = qy * qz;
        REAL xw = qx * qw, yw = qy * qw, zw = qz * qw;
        REAL sx = scale_mod * scales[3 * i], sy = scale_mod * scales[3 * i + 1], sz = scale_mod * scales[3 * i + 2];
        REAL m11 = sx * ((REAL)1 - (REAL)2 * (yy + zz)), m12 = sx * (REAL)2 * (qxy - zw), m13 = sx * (REAL)2 * (qxz + yw);
        REAL m21 = sy * (REAL)2 * (qxy + zw), m22 = sy * ((REAL)1 - (REAL)2 * (xx + zz)), m23 = sy * (REAL)2 * (qyz - xw);
        REAL m31 = sz * (REAL)2 * (qxz - yw), m32 = sz * (REAL)2 * (qyz + xw), m33 = sz * ((REAL)1 - (REAL)2 * (xx + yy));
        const REAL* g = dcov3D + 6 * i;
        REAL g11 = g[0], g12 = g[1], g13 = g[2], g22 = g[3], g23 = g[4], g33 = g[5];
        REAL a11 = (REAL)2 * (m11 * g11 + m12 * g12 + m13 * g13);
        REAL a12 = (REAL)2 * (m11 * g12 + m12 * g22 + m13 * g23);
        REAL a13 = (REAL)2 * (m11 * g13 + m12 * g23 + m13 * g33);
        REAL a21 = (REAL)2 * (m21 * g11 + m22 * g12 + m23 * g13);
        REAL a22 = (REAL)2 * (m21 * g12 + m22 * g22 + m23 * g23);
        REAL a23 = (REAL)2 * (m21 * g13 + m22 * g23 + m23 * g33);
        REAL a31 = (REAL)2 * (m31 * g11 + m32 * g12 + m33 * g13);
        REAL a32 = (REAL)2 * (m31 * g12 + m32 * g22 + m33 * g23);
        REAL a33 = (REAL)2 * (m31 * g13 + m32 * g23 + m33 * g33);
        dscale[3 * i] = ((REAL)1 - (REAL)2 * (yy + zz)) * a11 + (REAL)2 * (qxy - zw) * a12 + (REAL)2 * (qxz + yw) * a13;
        dscale[3 * i + 1] = (REAL)2 * (qxy + zw) * a21 + ((REAL)1 - (REAL)2 * (xx + zz)) * a22 + (REAL)2 * (qyz - xw) * a23;
        dscale[3 * i + 2] = (REAL)2 * (qxz - yw) * a31 + (REAL)2 * (qyz + xw) * a32 + ((REAL)1 - (REAL)2 * (xx + yy)) * a33;
        drot[4 * i] = (REAL)4 * (-sz * (a31 * yw - a32 * xw + a33 * qxy) + sy * (a21 * zw - a22 * qxz + a23 * yy) + sx * (a12 * zw - a13 * yw - a11 * qyz));
        drot[4 * i + 1] = (REAL)4 * (sz * (a31 * zw + a32 * zz - a33 * qyz) - sy * (a21 * yw + a22 * qxy + a23 * xx) + sx * (a12 * yy + a13 * zw + a11 * qxz));
        drot[4 * i + 2] = (REAL)4 * (-sz * (a31 * xx + a32 * xw + a33 * qxz) + sy * (a21 * zw + a22 * yy + a23 * yw) - sx * (a12 * xw + a13 * xx + a11 * qxy));
        drot[4 * i + 3] = (REAL)4 * (sz * (a31 * xw - a32 * xx + a33 * qxy) - sy * (a21 * qxz - a22 * zw + a23 * qyz) + sx * (a12 * qyz - a13 * zz + a11 * yy));
    }
}

void SFX(orc_backward_preprocess)(int P, int M, const float* means3D, const int32_t* radii,
                                  const float* sh, const uint8_t* clamped, const float* scales,
                                  const float* rots, REAL scale_mod, const float* view,
                                  const float* proj, const float* campos, const REAL* dmean2D,
                                  const REAL* dcolor, const REAL* ddepth, const REAL* dcov3D,
                                  REAL* dmean3D, REAL* dsh, REAL* dscale, REAL* drot)
{
    SFX(orc_backward_preprocess_ctx) c_ = {P, M, means3D, radii, sh, clamped, scales, rots, scale_mod, view, proj, campos, dmean2D, dcolor, ddepth, dcov3D, dmean3D, dsh, dscale, drot};
    orc_parallel_for(P, 4096, SFX(orc_backward_preprocess_part), &c_);
}


/* ------------------------------------------------------------------------ */
/* Backward, exact mode: the true derivative of the forward restated above. */
/* ------------------------------------------------------------------------ */
/* The reference backward differs from the derivative of its own forward
 * (low-pass +0.3 on the covariance, backward.cu:98-99; a 1.3*tan box clamp,
 * :58-70; colour-clamp masks although the forward stores the unclamped
 * colour, gaussianForwardPass.cu:263; SH_C2[2] = 0.3154 where the forward
 * uses 0.3, gaussianForwardPass.cu:23).  This mode differentiates exactly
 * what the forward computes: blend decisions are re-made with the forward's
 * own evaluation (gaussEval.h:13-28) and cut at the forward's last
 * contributor, so the set of blended pairs is the forward's.
 *
 * Outputs (caller zeroes):  dndc[P*3] (dL/dNDC x,y; z unused), dcolor[P*3],
 * dopac[P], dmean3D[P*3], dcov3D[P*6] (off-diagonals are derivatives w.r.t.
 * the single shared entry), dsh[P*M*3], dscale[P*3], drot[P*4].
 * T_final[H*W] is the forward's final transmittance. */
void SFX(orc_backward_exact)(const orc_cfg* cfg, int P,
                             const float* means3D, const float* scales, const float* rots,
                             const float* opac, const float* sh,
                             const uint32_t* ranges, const uint32_t* point_list,
                             const REAL* means2D, const REAL* cov2D, const REAL* cov3D,
                             const REAL* rgb, const REAL* depth, const int32_t* radii,
                             const REAL* T_final, const uint32_t* n_contrib,
                             const float* dL_dpix, const float* dL_ddepth, const float* dL_dalpha,
                             REAL* dndc, REAL* dcolor, REAL* dopac, REAL* dmean3D, REAL* dcov3D,
                             REAL* dsh, REAL* dscale, REAL* drot)
{
    const int W = cfg->W, H = cfg->H, gw = (W + 15) / 16;
    const REAL min_alpha = (REAL)(1.0f / 255.0f), max_alpha = (REAL)0.99f;
    double* gm2 = (double*)calloc((size_t)P * 2, sizeof(double));   /* dL/dmean2D (pixels) */
    double* gc2 = (double*)calloc((size_t)P * 3, sizeof(double));   /* dL/dcov2D */
    double* gop = (double*)calloc((size_t)P, sizeof(double));
    double* gcol = (double*)calloc((size_t)P * 3, sizeof(double));
    double* gdep = (double*)calloc((size_t)P, sizeof(double));
    uint32_t* ids = NULL; REAL* av = NULL; REAL* Tv = NULL; REAL* gv = NULL; uint8_t* uc = NULL;
    size_t cap = 0;
    for (int py = 0; py < H; ++py) {
        for (int px = 0; px < W; ++px) {
            int tile = (py / 16) * gw + (px / 16);
            uint32_t s = ranges[2 * tile], e = ranges[2 * tile + 1];
            size_t pix = (size_t)py * W + px;
            uint32_t last = n_contrib[pix];
            if (e - s > cap) {
                cap = e - s;
                ids = (uint32_t*)realloc(ids, cap * sizeof(uint32_t));
                av = (REAL*)realloc(av, cap * sizeof(REAL));
                Tv = (REAL*)realloc(Tv, cap * sizeof(REAL));
                gv = (REAL*)realloc(gv, cap * sizeof(REAL));
                uc = (uint8_t*)realloc(uc, cap);
            }
            /* forward replay: the blended list of this pixel */
            size_t n = 0;
            REAL T = 1;
            REAL qx = (REAL)px, qy = (REAL)py;
            for (uint32_t j = s; j < e && (j - s) < last; ++j) {
                uint32_t id = point_list[j];
                REAL det = SFX(blend_det)(cov2D + 3 * id);
                REAL g = SFX(gauss_eval)(means2D[2 * id], means2D[2 * id + 1], cov2D[3 * id],
                                         cov2D[3 * id + 1], cov2D[3 * id + 2], det, qx, qy);
                REAL og = (REAL)opac[id] * g;
                REAL a = og < max_alpha ? og : max_alpha;
                if (!(a >= min_alpha)) continue;
                ids[n] = id; av[n] = a; Tv[n] = T; gv[n] = g; uc[n] = og < max_alpha;
                T = T * ((REAL)1 - a);
                ++n;
            }
            REAL Tf = T_final[pix];
            double dLC[3], dLD = dL_ddepth[pix], dLA = dL_dalpha[pix];
            for (int c = 0; c < 3; ++c) dLC[c] = dL_dpix[(size_t)c * H * W + pix];
            double SC[3], SD = 0, SW = 0;
            for (int c = 0; c < 3; ++c) SC[c] = (double)Tf * cfg->bg[c];
            for (size_t k = n; k-- > 0;) {
                uint32_t id = ids[k];
                double a = av[k], Ti = Tv[k], g = gv[k];
                double ia = 1.0 / (1.0 - a);
                double dLda = 0;
                for (int c = 0; c < 3; ++c) {
                    double col = rgb[3 * id + c];
                    dLda += dLC[c] * (col * Ti - SC[c] * ia);
                    gcol[3 * id + c] += a * Ti * dLC[c];
                    SC[c] += col * a * Ti;
                }
                double dd = depth[id];
                dLda += dLD * (dd * Ti - SD * ia);
                gdep[id] += a * Ti * dLD;
                SD += dd * a * Ti;
                dLda += dLA * (Ti - SW * ia);
                SW += a * Ti;
                if (!uc[k]) continue; /* alpha clamped at 0.99: no dependence on o or g */
                gop[id] += dLda * g;
                double dLdg = dLda * (double)opac[id];
                double dLdm = dLdg * (-0.5 * g);
                double cxx = cov2D[3 * id], cxy = cov2D[3 * id + 1], cyy = cov2D[3 * id + 2];
                double det = cxx * cyy - cxy * cxy;
                double dx = (double)qx - means2D[2 * id], dy = (double)qy - means2D[2 * id + 1];
                double num = cyy * dx * dx - 2 * cxy * dx * dy + cxx * dy * dy;
                if (num / det < 0) continue; /* clamped to a constant in the forward */
                double dmddx = (2 * cyy * dx - 2 * cxy * dy) / det;
                double dmddy = (2 * cxx * dy - 2 * cxy * dx) / det;
                gm2[2 * id] += -dLdm * dmddx;
                gm2[2 * id + 1] += -dLdm * dmddy;
                double id2 = 1.0 / (det * det);
                gc2[3 * id] += dLdm * (dy * dy / det - num * cyy * id2);
                gc2[3 * id + 1] += dLdm * (-2 * dx * dy / det + 2 * num * cxy * id2);
                gc2[3 * id + 2] += dLdm * (dx * dx / det - num * cxx * id2);
            }
        }
    }
    free(ids); free(av); free(Tv); free(gv); free(uc);

    const float* V = cfg->view;
    const float* PM = cfg->proj;
    const double f = cfg->focal_x;
    const double L = (double)W / (2.0 * cfg->focal_x);
    const int M = cfg->M, deg = cfg->degree;
    for (int i = 0; i < P; ++i) {
        if (radii[i] <= 0) continue;
        double m[3] = {means3D[3 * i], means3D[3 * i + 1], means3D[3 * i + 2]};
        double gm[3] = {0, 0, 0};
        /* screen position and depth: ndc = clip.xyz / (clip.w + 1e-5) */
        double clip[4];
        for (int r = 0; r < 4; ++r)
            clip[r] = PM[r] * m[0] + PM[4 + r] * m[1] + PM[8 + r] * m[2] + PM[12 + r];
        double wi = 1.0 / (clip[3] + 1e-5);
        double gn[3] = {0.5 * W * gm2[2 * i], 0.5 * H * gm2[2 * i + 1], gdep[i]};
        dndc[3 * i] = (REAL)gn[0]; dndc[3 * i + 1] = (REAL)gn[1]; dndc[3 * i + 2] = 0;
        double gcl[4] = {gn[0] * wi, gn[1] * wi, gn[2] * wi,
                         -(gn[0] * clip[0] + gn[1] * clip[1] + gn[2] * clip[2]) * wi * wi};
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 4; ++r) gm[c] += PM[4 * c + r] * gcl[r];
        /* covariance chain */
        double t[3];
        for (int r = 0; r < 3; ++r) t[r] = V[r] * m[0] + V[4 + r] * m[1] + V[8 + r] * m[2] + V[12 + r];
        double rx = t[0] / t[2], ry = t[1] / t[2];
        double nn = sqrt(rx * rx + ry * ry) / L;
        int clampd = nn > 1.0;
        double txp = t[0], typ = t[1];
        if (clampd) { txp = rx / nn * t[2]; typ = ry / nn * t[2]; }
        double tz = t[2];
        double rgt[3] = {V[0], V[4], V[8]}, upv[3] = {V[1], V[5], V[9]}, fw[3] = {V[2], V[6], V[10]};
        double jx[3], jy[3];
        for (int k = 0; k < 3; ++k) {
            jx[k] = f * (rgt[k] / tz - txp * fw[k] / (tz * tz));
            jy[k] = f * (upv[k] / tz - typ * fw[k] / (tz * tz));
        }
        const REAL* pc = cov3D + 6 * i;
        double S[3][3] = {{pc[0], pc[1], pc[2]}, {pc[1], pc[3], pc[4]}, {pc[2], pc[4], pc[5]}};
        double gxx = gc2[3 * i], gxy = gc2[3 * i + 1], gyy = gc2[3 * i + 2];
        double Gf[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                Gf[a][b] = gxx * jx[a] * jx[b] + gyy * jy[a] * jy[b] + gxy * jx[a] * jy[b];
        double* dc = NULL;
        (void)dc;
        dcov3D[6 * i + 0] = (REAL)Gf[0][0];
        dcov3D[6 * i + 1] = (REAL)(Gf[0][1] + Gf[1][0]);
        dcov3D[6 * i + 2] = (REAL)(Gf[0][2] + Gf[2][0]);
        dcov3D[6 * i + 3] = (REAL)Gf[1][1];
        dcov3D[6 * i + 4] = (REAL)(Gf[1][2] + Gf[2][1]);
        dcov3D[6 * i + 5] = (REAL)Gf[2][2];
        double Sjx[3], Sjy[3];
        for (int a = 0; a < 3; ++a) {
            Sjx[a] = S[a][0] * jx[0] + S[a][1] * jx[1] + S[a][2] * jx[2];
            Sjy[a] = S[a][0] * jy[0] + S[a][1] * jy[1] + S[a][2] * jy[2];
        }
        double gjx[3], gjy[3];
        for (int a = 0; a < 3; ++a) {
            gjx[a] = 2 * gxx * Sjx[a] + gxy * Sjy[a];
            gjy[a] = 2 * gyy * Sjy[a] + gxy * Sjx[a];
        }
        double gtxp = 0, gtyp = 0, gtz = 0;
        for (int k = 0; k < 3; ++k) {
            gtxp += gjx[k] * (-f * fw[k] / (tz * tz));
            gtyp += gjy[k] * (-f * fw[k] / (tz * tz));
            gtz += gjx[k] * f * (-rgt[k] / (tz * tz) + 2 * txp * fw[k] / (tz * tz * tz));
            gtz += gjy[k] * f * (-upv[k] / (tz * tz) + 2 * typ * fw[k] / (tz * tz * tz));
        }
        double gt[3];
        if (!clampd) {
            gt[0] = gtxp; gt[1] = gtyp; gt[2] = gtz;
        } else {
            double r2 = t[0] * t[0] + t[1] * t[1], r1 = sqrt(r2), r3 = r2 * r1;
            double dxx = L * tz * t[1] * t[1] / r3, dxy = -L * tz * t[0] * t[1] / r3, dxz = L * t[0] / r1;
            double dyx = -L * tz * t[0] * t[1] / r3, dyy = L * tz * t[0] * t[0] / r3, dyz = L * t[1] / r1;
            gt[0] = gtxp * dxx + gtyp * dyx;
            gt[1] = gtxp * dxy + gtyp * dyy;
            gt[2] = gtz + gtxp * dxz + gtyp * dyz;
        }
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) gm[c] += V[4 * c + r] * gt[r];
        /* Sigma = M M^T, M = R diag(s) with R the rotation of q = (w, x, y, z) */
        const float* q = rots + 4 * i;
        double w = q[0], x = q[1], y = q[2], z = q[3];
        double R[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)},
                          {2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)},
                          {2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)}};
        double s[3] = {scales[3 * i], scales[3 * i + 1], scales[3 * i + 2]};
        double Gs[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) Gs[a][b] = 0.5 * (Gf[a][b] + Gf[b][a]);
        double dM[3][3];
        for (int a = 0; a < 3; ++a)
            for (int k = 0; k < 3; ++k) {
                double acc = 0;
                for (int b = 0; b < 3; ++b) acc += Gs[a][b] * R[b][k] * s[k];
                dM[a][k] = 2 * acc;
            }
        for (int k = 0; k < 3; ++k) {
            double acc = 0;
            for (int a = 0; a < 3; ++a) acc += dM[a][k] * R[a][k];
            dscale[3 * i + k] = (REAL)acc;
        }
        double dR[3][3];
        for (int a = 0; a < 3; ++a)
            for (int k = 0; k < 3; ++k) dR[a][k] = dM[a][k] * s[k];
        double gw_ = dR[0][1] * (-2 * z) + dR[0][2] * (2 * y) + dR[1][0] * (2 * z) + dR[1][2] * (-2 * x) +
                     dR[2][0] * (-2 * y) + dR[2][1] * (2 * x);
        double gx = dR[0][1] * (2 * y) + dR[0][2] * (2 * z) + dR[1][0] * (2 * y) + dR[1][1] * (-4 * x) +
                    dR[1][2] * (-2 * w) + dR[2][0] * (2 * z) + dR[2][1] * (2 * w) + dR[2][2] * (-4 * x);
        double gy = dR[0][0] * (-4 * y) + dR[0][1] * (2 * x) + dR[0][2] * (2 * w) + dR[1][0] * (2 * x) +
                    dR[1][2] * (2 * z) + dR[2][0] * (-2 * w) + dR[2][1] * (2 * z) + dR[2][2] * (-4 * y);
        double gz = dR[0][0] * (-4 * z) + dR[0][1] * (-2 * w) + dR[0][2] * (2 * x) + dR[1][0] * (2 * w) +
                    dR[1][1] * (-4 * z) + dR[1][2] * (2 * y) + dR[2][0] * (2 * x) + dR[2][1] * (2 * y);
        drot[4 * i] = (REAL)gw_; drot[4 * i + 1] = (REAL)gx; drot[4 * i + 2] = (REAL)gy; drot[4 * i + 3] = (REAL)gz;
        /* colour: rgb = sum_k basis_k(dir) sh_k + 0.5, dir = (m - campos)/|m - campos| */
        double v[3] = {m[0] - cfg->campos[0], m[1] - cfg->campos[1], m[2] - cfg->campos[2]};
        double vn = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        double X = v[0] / vn, Y = v[1] / vn, Z = v[2] / vn;
        double gcl3[3] = {gcol[3 * i], gcol[3 * i + 1], gcol[3 * i + 2]};
        dcolor[3 * i] = (REAL)gcl3[0]; dcolor[3 * i + 1] = (REAL)gcl3[1]; dcolor[3 * i + 2] = (REAL)gcl3[2];
        dopac[i] = (REAL)gop[i];
        const double C1 = 0.4886025119029199f, C2a = 1.0925484305920792f, C2e = 0.5462742152960396f;
        const double C30 = 0.5900435899266435f, C31 = 2.890611442640554f, C32 = 0.4570457994644658f;
        const double C33 = 0.3731763325901154f, C35 = 1.445305721320277f;
        double b[16], db[16][3];
        memset(db, 0, sizeof(db));
        double xx = X * X, yy = Y * Y, zz = Z * Z;
        b[0] = 0.28209479177387814f;
        b[1] = -C1 * Y; db[1][1] = -C1;
        b[2] = C1 * Z; db[2][2] = C1;
        b[3] = -C1 * X; db[3][0] = -C1;
        b[4] = C2a * X * Y; db[4][0] = C2a * Y; db[4][1] = C2a * X;
        b[5] = -C2a * Y * Z; db[5][1] = -C2a * Z; db[5][2] = -C2a * Y;
        b[6] = 0.3f * (2 * zz - xx - yy); db[6][0] = -2 * 0.3f * X; db[6][1] = -2 * 0.3f * Y; db[6][2] = 4 * 0.3f * Z;
        b[7] = -C2a * X * Z; db[7][0] = -C2a * Z; db[7][2] = -C2a * X;
        b[8] = C2e * (xx - yy); db[8][0] = 2 * C2e * X; db[8][1] = -2 * C2e * Y;
        b[9] = -C30 * Y * (3 * xx - yy); db[9][0] = -6 * C30 * X * Y; db[9][1] = -C30 * (3 * xx - 3 * yy);
        b[10] = C31 * X * Y * Z; db[10][0] = C31 * Y * Z; db[10][1] = C31 * X * Z; db[10][2] = C31 * X * Y;
        b[11] = -C32 * Y * (4 * zz - xx - yy); db[11][0] = 2 * C32 * X * Y; db[11][1] = -C32 * (4 * zz - xx - 3 * yy); db[11][2] = -8 * C32 * Y * Z;
        b[12] = C33 * Z * (2 * zz - 3 * xx - 3 * yy); db[12][0] = -6 * C33 * X * Z; db[12][1] = -6 * C33 * Y * Z; db[12][2] = C33 * (6 * zz - 3 * xx - 3 * yy);
        b[13] = -C32 * X * (4 * zz - xx - yy); db[13][0] = -C32 * (4 * zz - 3 * xx - yy); db[13][1] = 2 * C32 * X * Y; db[13][2] = -8 * C32 * X * Z;
        b[14] = C35 * Z * (xx - yy); db[14][0] = 2 * C35 * X * Z; db[14][1] = -2 * C35 * Y * Z; db[14][2] = C35 * (xx - yy);
        b[15] = -C30 * X * (xx - 3 * yy); db[15][0] = -C30 * (3 * xx - 3 * yy); db[15][1] = 6 * C30 * X * Y;
        /* bands the forward evaluated: degree d needs (d+1)^2 coefficients */
        int de = deg > 3 ? 3 : deg;
        while (de > 0 && (de + 1) * (de + 1) > M) --de;
        int nb = (de + 1) * (de + 1);
        double gdir[3] = {0, 0, 0};
        const float* sdat = sh + (size_t)i * M * 3;
        for (int k = 0; k < nb; ++k)
            for (int c = 0; c < 3; ++c) {
                dsh[((size_t)i * M + k) * 3 + c] = (REAL)(b[k] * gcl3[c]);
                for (int a = 0; a < 3; ++a) gdir[a] += sdat[3 * k + c] * db[k][a] * gcl3[c];
            }
        double dd[3] = {X, Y, Z};
        for (int a = 0; a < 3; ++a) {
            double acc = 0;
            for (int bb = 0; bb < 3; ++bb) acc += ((a == bb ? 1.0 : 0.0) - dd[a] * dd[bb]) * gdir[bb];
            gm[a] += acc / vn;
        }
        dmean3D[3 * i] = (REAL)gm[0]; dmean3D[3 * i + 1] = (REAL)gm[1]; dmean3D[3 * i + 2] = (REAL)gm[2];
    }
    free(gm2); free(gc2); free(gop); free(gcol); free(gdep);
}
