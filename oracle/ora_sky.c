/* Oracle: the medium, its majorant octrees and ray traversal.
 * TEST INFRASTRUCTURE ONLY (see ora.h).
 *
 * Restates the services the reference takes from htsky 0.3 / star-vx 0.3
 * (not vendored; call sites src/atmosphere/htrdr_atmosphere_compute_radiance_sw.c:87,
 * 130, 163-166, 202, 243, 369, 427-429 and ..._lw.c:78, 113-115, 205):
 *   - htsky_fetch_raw_property   -> site_k()
 *   - htsky_fetch_svx_voxel_property(SVX_MIN/SVX_MAX) -> the leaf {kmin,kmax}
 *   - htsky_trace_ray + hit filter -> ora_trace_ray()
 *   - htsky_find_spectral_band / htsky_spectral_band_sample_quadrature
 * with the definitions spelled out next to each function. */
#include "ora_internal.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/*******************************************************************************
 * Spectral bands and quadrature (htsky_find_spectral_band and
 * htsky_spectral_band_sample_quadrature; called from
 * src/atmosphere/htrdr_atmosphere_draw_map.c:176-177, 262-263, 383-384)
 ******************************************************************************/
/* Band i such that lo[i] <= wlen < hi[i]; a wavelength equal to the upper
 * bound of the last band maps to it.  Returns nbands when none matches. */
size_t
ora_find_band(const struct ora_scene* scn, double wlen)
{
  size_t lo = 0, hi = scn->nbands;
  while(lo < hi) { /* first band whose upper bound is > wlen */
    const size_t mid = lo + (hi - lo) / 2;
    if(scn->band_hi[mid] <= wlen) lo = mid + 1; else hi = mid;
  }
  if(lo == scn->nbands) {
    if(scn->nbands && wlen == scn->band_hi[scn->nbands - 1]) return scn->nbands - 1;
    return scn->nbands;
  }
  return wlen >= scn->band_lo[lo] ? lo : scn->nbands;
}

/* First quadrature point whose cumulative weight is > r. */
size_t
ora_sample_quad(const struct ora_scene* scn, double r, size_t iband)
{
  const double* cum = scn->quad_cum + scn->quad_off[iband];
  const size_t n = scn->nquads[iband];
  size_t lo = 0, hi = n;
  while(lo < hi) {
    const size_t mid = lo + (hi - lo) / 2;
    if(cum[mid] <= r) lo = mid + 1; else hi = mid;
  }
  return lo < n ? lo : n - 1;
}

/*******************************************************************************
 * Medium: gas layers and cloud cells
 ******************************************************************************/
/* Layer i with z_i <= z < z_{i+1}, clamped to the column. */
int
ora_layer_of(const struct ora_scene* scn, double z)
{
  size_t lo = 0, hi = scn->nlayers + 1;
  while(lo < hi) { /* upper_bound */
    const size_t mid = lo + (hi - lo) / 2;
    if(scn->layer_z[mid] <= z) lo = mid + 1; else hi = mid;
  }
  if(lo == 0) return 0;
  if(lo > scn->nlayers) return (int)scn->nlayers - 1;
  return (int)lo - 1;
}

static float
gas_k(const struct ora_scene* scn, uint32_t q, int prop, int layer)
{
  const size_t i = (size_t)q * scn->nlayers + (size_t)layer;
  switch(prop) {
    case ORA_KA: return scn->gas_ka[i];
    case ORA_KS: return scn->gas_ks[i];
    default: return scn->gas_kext[i];
  }
}

/* k of the cloud cell for a property: lwc * sigma_prop (single precision). */
static float
cloud_k(const struct ora_scene* scn, uint32_t band, int prop, size_t cell)
{
  const float lwc = scn->lwc[cell];
  const float sig = scn->sig[band * 3 + (uint32_t)prop];
  return lwc * sig;
}

/* Raw k at a collision site: cloud cell (if any) plus the gas layer.  The
 * sum is computed in single precision exactly as the majorant build does, so
 * that k lies inside the [kmin, kmax] of the leaf holding the site.  cpnt:
 * 1 gas only, 2 particles only, 3 both (HTSKY_CPNT_FLAG_GAS/PARTICLES). */
double
ora_site_k(const struct ora_scene* scn, const struct ora_site* s, uint32_t band, uint32_t q,
           int prop, int cpnt)
{
  float kc = 0.f, kg = 0.f;
  if((cpnt & 2) && s->cell >= 0) kc = cloud_k(scn, band, prop, (size_t)s->cell);
  if((cpnt & 1) && s->layer >= 0) kg = gas_k(scn, q, prop, s->layer);
  return (double)(kc + kg);
}

/*******************************************************************************
 * Majorant octrees.  One octree per (band, quadrature point, property) over
 * the cloud cell grid, each node a packed {kmin, kmax, first child} record.
 *
 *  - level 0 (cell): k_cloud + [min, max] of the gas over the layers that
 *    overlap the cell's z-extent;
 *  - level L > 0 covers 2^L cells per axis (root: 2^D >= max(nx, ny, nz));
 *    min/max over its valid children;
 *  - a node is a leaf when all its valid children are leaves and either
 *    L <= L_force (the -V maximum definition of the structure) or
 *    (kmax - kmin) * 2^L * max(dx, dy, dz) <= optical_thickness (-T);
 *  - nodes are stored breadth first; an internal node's 8 children are
 *    contiguous in octant order (bit 0: x, bit 1: y, bit 2: z).  Children
 *    outside the grid are stored as empty leaves.
 * This is the structure htsky builds per (band, quadrature point) (see
 * doc/htrdr-atmosphere.1.in:221-230, 403-418); its exact merge rule is not in
 * the reference tree, so the rule above is the definition both sides use.
 ******************************************************************************/
struct level {
  uint32_t n[3];
  float* kmin;
  float* kmax;
  uint8_t* leaf;
};

static int
build_tree(struct ora_scene* scn, uint32_t band, uint32_t q, int prop, struct ora_tree* tree)
{
  const uint32_t D = scn->depth;
  struct level* lv = calloc(D + 1, sizeof(struct level));
  const double cmax = fmax(scn->cell[0], fmax(scn->cell[1], scn->cell[2]));
  uint32_t L;
  size_t n_internal = 0, total, count, idx;
  uint32_t* coord = NULL; /* L | i | j | k per node during emission */
  int res = ORA_RES_OK;
  if(!lv) return ORA_RES_MEM_ERR;

  for(L = 0; L <= D; ++L) {
    size_t nn;
    int a;
    for(a = 0; a < 3; ++a) lv[L].n[a] = (scn->def[a] + (1u << L) - 1) >> L;
    nn = (size_t)lv[L].n[0] * lv[L].n[1] * lv[L].n[2];
    lv[L].kmin = malloc(nn * sizeof(float));
    lv[L].kmax = malloc(nn * sizeof(float));
    lv[L].leaf = malloc(nn);
    if(!lv[L].kmin || !lv[L].kmax || !lv[L].leaf) { res = ORA_RES_MEM_ERR; goto exit; }
  }

  { /* Level 0: the cloud cells */
    uint32_t i, j, k;
    for(k = 0; k < scn->def[2]; ++k) {
      const int l0 = scn->cell_layer_lo[k], l1 = scn->cell_layer_hi[k];
      float gmin = 0.f, gmax = 0.f;
      int l;
      if(l0 >= 0) {
        gmin = gmax = gas_k(scn, q, prop, l0);
        for(l = l0 + 1; l <= l1; ++l) {
          const float g = gas_k(scn, q, prop, l);
          if(g < gmin) gmin = g;
          if(g > gmax) gmax = g;
        }
      }
      for(j = 0; j < scn->def[1]; ++j) {
        for(i = 0; i < scn->def[0]; ++i) {
          const size_t c = ((size_t)k * scn->def[1] + j) * scn->def[0] + i;
          const float kc = cloud_k(scn, band, prop, c);
          lv[0].kmin[c] = kc + gmin;
          lv[0].kmax[c] = kc + gmax;
          lv[0].leaf[c] = 1;
        }
      }
    }
  }

  for(L = 1; L <= D; ++L) { /* Bottom-up min/max and merge decision */
    const struct level* c = &lv[L - 1];
    struct level* p = &lv[L];
    const double size = (double)(1u << L) * cmax;
    uint32_t i, j, k;
    for(k = 0; k < p->n[2]; ++k)
    for(j = 0; j < p->n[1]; ++j)
    for(i = 0; i < p->n[0]; ++i) {
      const size_t pi = ((size_t)k * p->n[1] + j) * p->n[0] + i;
      float mn = FLT_MAX, mx = -FLT_MAX;
      int all_leaf = 1, oct;
      for(oct = 0; oct < 8; ++oct) {
        const uint32_t ci = 2 * i + (oct & 1), cj = 2 * j + ((oct >> 1) & 1);
        const uint32_t ck = 2 * k + (oct >> 2);
        size_t cc;
        if(ci >= c->n[0] || cj >= c->n[1] || ck >= c->n[2]) continue;
        cc = ((size_t)ck * c->n[1] + cj) * c->n[0] + ci;
        if(c->kmin[cc] < mn) mn = c->kmin[cc];
        if(c->kmax[cc] > mx) mx = c->kmax[cc];
        all_leaf &= c->leaf[cc];
      }
      p->kmin[pi] = mn;
      p->kmax[pi] = mx;
      p->leaf[pi] = (uint8_t)(all_leaf
        && (L <= scn->level_force || ((double)mx - (double)mn) * size <= scn->tau_thresh));
      if(!p->leaf[pi]) ++n_internal;
    }
  }

  total = 1 + 8 * n_internal;
  tree->nodes = malloc(total * sizeof(struct ora_node));
  coord = malloc(total * 4 * sizeof(uint32_t));
  if(!tree->nodes || !coord) { res = ORA_RES_MEM_ERR; goto exit; }

  /* Breadth-first emission */
  tree->nodes[0].kmin = lv[D].kmin[0];
  tree->nodes[0].kmax = lv[D].kmax[0];
  tree->nodes[0].pad = 0;
  coord[0] = D; coord[1] = coord[2] = coord[3] = 0;
  count = 1;
  for(idx = 0; idx < count; ++idx) {
    const uint32_t Ln = coord[idx * 4 + 0];
    const uint32_t i = coord[idx * 4 + 1], j = coord[idx * 4 + 2], k = coord[idx * 4 + 3];
    const struct level* p = &lv[Ln == 0xFFFFFFFFu ? 0 : Ln];
    int oct;
    if(Ln == 0xFFFFFFFFu) { tree->nodes[idx].child = ORA_LEAF; continue; } /* empty */
    if(p->leaf[((size_t)k * p->n[1] + j) * p->n[0] + i]) {
      tree->nodes[idx].child = ORA_LEAF;
      continue;
    }
    tree->nodes[idx].child = (uint32_t)count;
    for(oct = 0; oct < 8; ++oct) {
      const struct level* c = &lv[Ln - 1];
      const uint32_t ci = 2 * i + (oct & 1), cj = 2 * j + ((oct >> 1) & 1);
      const uint32_t ck = 2 * k + (oct >> 2);
      struct ora_node* nd = &tree->nodes[count];
      uint32_t* cd = &coord[count * 4];
      nd->pad = 0;
      if(ci >= c->n[0] || cj >= c->n[1] || ck >= c->n[2]) {
        nd->kmin = nd->kmax = 0.f;
        nd->child = ORA_LEAF;
        cd[0] = 0xFFFFFFFFu;
      } else {
        const size_t cc = ((size_t)ck * c->n[1] + cj) * c->n[0] + ci;
        nd->kmin = c->kmin[cc];
        nd->kmax = c->kmax[cc];
        cd[0] = Ln - 1; cd[1] = ci; cd[2] = cj; cd[3] = ck;
      }
      ++count;
    }
  }
  tree->n = count;

exit:
  for(L = 0; L <= D; ++L) { free(lv[L].kmin); free(lv[L].kmax); free(lv[L].leaf); }
  free(lv);
  free(coord);
  return res;
}

/* Descend from the root to the leaf holding the (valid) cell; bit-exact
 * integer work shared with the CUDA traversal. */
int
ora_locate_leaf(const struct ora_scene* scn, uint32_t iband, uint32_t iquad, int prop,
                const uint32_t cell[3], uint32_t* node, uint32_t* level)
{
  const struct ora_tree* t;
  uint32_t q, n = 0, L;
  if(!scn->has_cloud || iband >= scn->nbands || iquad >= scn->nquads[iband]) return ORA_RES_BAD_ARG;
  if(cell[0] >= scn->def[0] || cell[1] >= scn->def[1] || cell[2] >= scn->def[2]) return ORA_RES_BAD_ARG;
  q = (uint32_t)scn->quad_off[iband] + iquad;
  t = &scn->trees[(size_t)q * 3 + (size_t)prop];
  if(!t->nodes) return ORA_RES_BAD_OP;
  L = scn->depth;
  while(t->nodes[n].child != ORA_LEAF) {
    uint32_t oct;
    --L;
    oct = ((cell[0] >> L) & 1u) | (((cell[1] >> L) & 1u) << 1) | (((cell[2] >> L) & 1u) << 2);
    n = t->nodes[n].child + oct;
  }
  *node = n;
  *level = L;
  return ORA_RES_OK;
}

size_t
ora_scene_tree(const struct ora_scene* scn, uint32_t iband, uint32_t iquad, int prop,
               const struct ora_node** nodes)
{
  const struct ora_tree* t;
  if(!scn->has_cloud || iband >= scn->nbands || iquad >= scn->nquads[iband]) { *nodes = NULL; return 0; }
  t = &scn->trees[((size_t)scn->quad_off[iband] + iquad) * 3 + (size_t)prop];
  *nodes = t->nodes;
  return t->n;
}

uint32_t
ora_scene_tree_depth(const struct ora_scene* scn) { return scn->depth; }

/*******************************************************************************
 * Scene creation
 ******************************************************************************/
static void
onb(const double n[3], double b1[3], double b2[3])
{
  /* T. Duff et al., "Building an Orthonormal Basis, Revisited", JCGT 6(1) 2017 */
  const double sign = copysign(1.0, n[2]);
  const double a = -1.0 / (sign + n[2]);
  const double b = n[0] * n[1] * a;
  b1[0] = 1.0 + sign * n[0] * n[0] * a; b1[1] = sign * b; b1[2] = -sign * n[0];
  b2[0] = b; b2[1] = sign + n[1] * n[1] * a; b2[2] = -n[1];
}

void
ora_onb(const double n[3], double b1[3], double b2[3]) { onb(n, b1, b2); }

int
ora_scene_create(const struct ora_scene_desc* d, struct ora_scene** out)
{
  struct ora_scene* s = calloc(1, sizeof(*s));
  size_t nq = 0, i, ncells = 0;
  int a;
  if(!s) return ORA_RES_MEM_ERR;
  if(!d->nlayers || !d->nbands) { free(s); return ORA_RES_BAD_ARG; }
  s->nlayers = d->nlayers;
  s->nbands = d->nbands;
  for(i = 0; i < d->nbands; ++i) nq += d->nquads[i];
  s->nq_total = nq;
  s->layer_z = malloc((d->nlayers + 1) * sizeof(double));
  s->layer_T = malloc(d->nlayers * sizeof(float));
  s->band_lo = malloc(d->nbands * sizeof(double));
  s->band_hi = malloc(d->nbands * sizeof(double));
  s->nquads = malloc(d->nbands * sizeof(uint32_t));
  s->quad_off = malloc((d->nbands + 1) * sizeof(size_t));
  s->quad_cum = malloc(nq * sizeof(double));
  s->gas_ka = malloc(nq * d->nlayers * sizeof(float));
  s->gas_ks = malloc(nq * d->nlayers * sizeof(float));
  s->gas_kext = malloc(nq * d->nlayers * sizeof(float));
  s->sig = malloc(d->nbands * 3 * sizeof(float));
  s->cloud_g = malloc(d->nbands * sizeof(float));
  memcpy(s->layer_z, d->layer_z, (d->nlayers + 1) * sizeof(double));
  memcpy(s->layer_T, d->layer_T, d->nlayers * sizeof(float));
  memcpy(s->band_lo, d->band_lo, d->nbands * sizeof(double));
  memcpy(s->band_hi, d->band_hi, d->nbands * sizeof(double));
  memcpy(s->nquads, d->nquads, d->nbands * sizeof(uint32_t));
  memcpy(s->gas_ka, d->gas_ka, nq * d->nlayers * sizeof(float));
  memcpy(s->gas_ks, d->gas_ks, nq * d->nlayers * sizeof(float));
  for(i = 0; i < nq * d->nlayers; ++i) s->gas_kext[i] = s->gas_ka[i] + s->gas_ks[i];
  s->quad_off[0] = 0;
  for(i = 0; i < d->nbands; ++i) {
    size_t iq;
    double acc = 0;
    s->quad_off[i + 1] = s->quad_off[i] + d->nquads[i];
    for(iq = 0; iq < d->nquads[i]; ++iq) {
      acc += d->quad_w[s->quad_off[i] + iq];
      s->quad_cum[s->quad_off[i] + iq] = acc;
    }
    s->quad_cum[s->quad_off[i + 1] - 1] = 1.0;
  }
  for(i = 0; i < d->nbands; ++i) {
    const double se = d->cloud_sigma_ext ? (double)d->cloud_sigma_ext[i] : 0.0;
    const double ssa = d->cloud_ssa ? (double)d->cloud_ssa[i] : 0.0;
    s->sig[i * 3 + ORA_KA] = (float)(se * (1.0 - ssa));
    s->sig[i * 3 + ORA_KS] = (float)(se * ssa);
    s->sig[i * 3 + ORA_KEXT] = (float)se;
    s->cloud_g[i] = d->cloud_g ? d->cloud_g[i] : 0.f;
  }
  s->ztop = s->layer_z[s->nlayers];

  s->has_cloud = d->cloud_def[0] && d->cloud_def[1] && d->cloud_def[2] && d->cloud_lwc;
  for(a = 0; a < 3; ++a) {
    s->def[a] = s->has_cloud ? d->cloud_def[a] : 0;
    s->lower[a] = d->cloud_lower[a];
    s->cell[a] = d->cloud_cell[a];
    s->upper[a] = s->lower[a] + (double)s->def[a] * s->cell[a];
  }
  s->repeat = d->repeat_clouds;
  s->tau_thresh = d->optical_thickness;
  if(s->has_cloud) {
    uint32_t mx = s->def[0];
    uint32_t k;
    if(s->def[1] > mx) mx = s->def[1];
    if(s->def[2] > mx) mx = s->def[2];
    s->depth = 0;
    while((1u << s->depth) < mx) ++s->depth;
    s->level_force = 0;
    for(a = 0; a < 3; ++a) {
      const uint32_t V = d->grid_max_definition[a];
      if(V && V < s->def[a]) {
        const uint32_t need = (s->def[a] + V - 1) / V;
        uint32_t Lf = 0;
        while((1u << Lf) < need) ++Lf;
        if(Lf > s->level_force) s->level_force = Lf;
      }
    }
    ncells = (size_t)s->def[0] * s->def[1] * s->def[2];
    s->lwc = malloc(ncells * sizeof(float));
    memcpy(s->lwc, d->cloud_lwc, ncells * sizeof(float));
    s->cell_layer_lo = malloc(s->def[2] * sizeof(int));
    s->cell_layer_hi = malloc(s->def[2] * sizeof(int));
    for(k = 0; k < s->def[2]; ++k) {
      const double zlo = s->lower[2] + (double)k * s->cell[2];
      const double zhi = zlo + s->cell[2];
      int l, lo = -1, hi = -1;
      for(l = 0; l < (int)s->nlayers; ++l) {
        if(s->layer_z[l] < zhi && s->layer_z[l + 1] > zlo) {
          if(lo < 0) lo = l;
          hi = l;
        }
      }
      s->cell_layer_lo[k] = lo;
      s->cell_layer_hi[k] = hi;
    }
    s->trees = calloc(nq * 3, sizeof(struct ora_tree));
    for(i = 0; i < d->nbands; ++i) {
      size_t iq;
      for(iq = 0; iq < d->nquads[i]; ++iq) {
        int p;
        for(p = 0; p < 3; ++p) {
          int r;
          if(!(d->props_mask & (1u << p))) continue;
          r = build_tree(s, (uint32_t)i, (uint32_t)(s->quad_off[i] + iq), p,
                         &s->trees[(s->quad_off[i] + iq) * 3 + (size_t)p]);
          if(r != ORA_RES_OK) { ora_scene_release(s); return r; }
        }
      }
    }
  }

  s->has_ground = d->has_ground;
  s->ground_brdf = d->ground_brdf;
  s->ground_reflectivity = d->ground_reflectivity;
  s->ground_temperature = d->ground_temperature;
  if(ora_ground_setup(s, d)) { ora_scene_release(s); return ORA_RES_MEM_ERR; }
  { /* Sun (src/atmosphere/htrdr_atmosphere_sun.c:66-101, htrdr_atmosphere.c:360-364) */
    const double az = d->sun_azimuth * M_PI / 180.0, el = d->sun_elevation * M_PI / 180.0;
    s->sun_dir[0] = cos(el) * cos(az);
    s->sun_dir[1] = cos(el) * sin(az);
    s->sun_dir[2] = sin(el);
    onb(s->sun_dir, s->sun_b1, s->sun_b2);
    s->sun_cos_half = cos(4.6524e-3);
    s->sun_solid_angle = 2.0 * M_PI * (1.0 - s->sun_cos_half);
    s->sun_temperature = 5778.0;
  }
  *out = s;
  return ORA_RES_OK;
}

void
ora_scene_release(struct ora_scene* s)
{
  size_t i;
  if(!s) return;
  if(s->trees) {
    for(i = 0; i < s->nq_total * 3; ++i) free(s->trees[i].nodes);
    free(s->trees);
  }
  free(s->layer_z); free(s->layer_T); free(s->band_lo); free(s->band_hi);
  free(s->nquads); free(s->quad_off); free(s->quad_cum); free(s->gas_ka); free(s->gas_ks);
  free(s->gas_kext); free(s->sig); free(s->cloud_g); free(s->lwc);
  free(s->cell_layer_lo); free(s->cell_layer_hi);
  ora_ground_release(s);
  free(s);
}

/*******************************************************************************
 * Traversal (htsky_trace_ray).  The ray [range0, range1] is clipped to the
 * gas column 0 <= z <= ztop and to 1e9 m (the give-up distance of
 * ..._sw.c:123).  Outside the cloud box (or the cloud slab when the clouds
 * repeat along X and Y) the medium is the gas layers, whose "voxels" are the
 * layer crossings with kmin = kmax = k_gas; inside it the leaves of the
 * property's octree are visited in order.  The filter gets each voxel with
 * its distance range clipped to the ray range, like an svx_hit.
 ******************************************************************************/
static void
slab(double o, double d, double lo, double hi, double* t0, double* t1)
{
  if(d != 0.0) {
    double a = (lo - o) / d, b = (hi - o) / d;
    if(a > b) { const double t = a; a = b; b = t; }
    if(a > *t0) *t0 = a;
    if(b < *t1) *t1 = b;
  } else if(o < lo || o > hi) {
    *t0 = 1; *t1 = 0; /* empty */
  }
}

static int64_t
floordiv(int64_t a, int64_t b)
{
  int64_t q = a / b;
  if((a % b != 0) && ((a < 0) != (b < 0))) --q;
  return q;
}

#define ORA_MAX_SEGS (1u << 24)

static int
trace_gas(const struct ora_scene* scn, uint32_t q, int prop, const double o[3], const double d[3],
          double ta, double tb, ora_filter_T filter, void* ctx, struct ora_counters* cnt,
          struct ora_seg* out_seg)
{
  int layer;
  const double z = o[2] + ta * d[2];
  uint32_t guard = 0;
  layer = ora_layer_of(scn, z);
  if(d[2] < 0 && layer > 0 && z <= scn->layer_z[layer]) --layer;
  while(ta < tb && guard++ < ORA_MAX_SEGS) {
    double tn = DBL_MAX, t1;
    if(d[2] > 0) tn = (scn->layer_z[layer + 1] - o[2]) / d[2];
    else if(d[2] < 0) tn = (scn->layer_z[layer] - o[2]) / d[2];
    t1 = tn < tb ? tn : tb;
    if(t1 < ta) t1 = ta;
    if(t1 > ta) {
      struct ora_seg seg;
      const double k = (double)gas_k(scn, q, prop, layer);
      seg.distance[0] = ta;
      seg.distance[1] = t1;
      seg.kmin = seg.kmax = k;
      seg.in_cloud = 0;
      seg.layer = layer;
      if(cnt) cnt->nseg++;
      if(!filter(&seg, o, d, ctx)) { *out_seg = seg; return 1; }
    }
    if(tn >= tb) break;
    ta = t1;
    layer += d[2] > 0 ? 1 : -1;
    if(layer < 0 || layer >= (int)scn->nlayers) break;
  }
  return 0;
}

static int
trace_cloud(const struct ora_scene* scn, uint32_t q, int prop, const double o[3],
            const double d[3], double ta, double tb, ora_filter_T filter, void* ctx,
            struct ora_counters* cnt, struct ora_seg* out_seg)
{
  const struct ora_tree* tree = &scn->trees[(size_t)q * 3 + (size_t)prop];
  int64_t tile[2] = {0, 0};
  uint32_t c[3];
  uint32_t guard = 0;
  int a;
  { /* Entry cell */
    double p[3];
    for(a = 0; a < 3; ++a) p[a] = o[a] + ta * d[a];
    for(a = 0; a < 3; ++a) {
      int64_t g = (int64_t)floor((p[a] - scn->lower[a]) / scn->cell[a]);
      if(scn->repeat && a < 2) {
        tile[a] = floordiv(g, (int64_t)scn->def[a]);
        g -= tile[a] * (int64_t)scn->def[a];
      }
      if(g < 0) g = 0;
      if(g >= (int64_t)scn->def[a]) g = scn->def[a] - 1;
      c[a] = (uint32_t)g;
    }
  }
  while(guard++ < ORA_MAX_SEGS) {
    uint32_t n = 0, L = scn->depth, lo[3], hi[3];
    double texit = DBL_MAX, t1;
    int axis = -1;
    if(cnt) cnt->nnode++;
    while(tree->nodes[n].child != ORA_LEAF) {
      uint32_t oct;
      --L;
      oct = ((c[0] >> L) & 1u) | (((c[1] >> L) & 1u) << 1) | (((c[2] >> L) & 1u) << 2);
      n = tree->nodes[n].child + oct;
      if(cnt) cnt->nnode++;
    }
    for(a = 0; a < 3; ++a) {
      const double off = (a < 2 ? (double)tile[a] * (double)scn->def[a] : 0.0);
      double wlo, whi, ta_;
      lo[a] = (c[a] >> L) << L;
      hi[a] = lo[a] + (1u << L);
      if(hi[a] > scn->def[a]) hi[a] = scn->def[a];
      wlo = scn->lower[a] + (off + (double)lo[a]) * scn->cell[a];
      whi = scn->lower[a] + (off + (double)hi[a]) * scn->cell[a];
      if(d[a] > 0) ta_ = (whi - o[a]) / d[a];
      else if(d[a] < 0) ta_ = (wlo - o[a]) / d[a];
      else continue;
      if(ta_ < texit) { texit = ta_; axis = a; }
    }
    t1 = texit < tb ? texit : tb;
    if(t1 < ta) t1 = ta;
    if(t1 > ta) {
      struct ora_seg seg;
      seg.distance[0] = ta;
      seg.distance[1] = t1;
      seg.kmin = (double)tree->nodes[n].kmin;
      seg.kmax = (double)tree->nodes[n].kmax;
      seg.in_cloud = 1;
      seg.layer = -1;
      for(a = 0; a < 3; ++a) { seg.lo[a] = lo[a]; seg.hi[a] = hi[a]; }
      seg.tile[0] = tile[0]; seg.tile[1] = tile[1];
      if(cnt) cnt->nseg++;
      if(!filter(&seg, o, d, ctx)) { *out_seg = seg; return 1; }
    }
    if(texit >= tb || axis < 0) break;
    { /* Next cell: exit face on `axis', the point's cell on the others */
      double p[3];
      int64_t nc;
      for(a = 0; a < 3; ++a) p[a] = o[a] + texit * d[a];
      for(a = 0; a < 3; ++a) {
        const int64_t off = (a < 2 ? tile[a] * (int64_t)scn->def[a] : 0);
        int64_t g;
        if(a == axis) continue;
        g = (int64_t)floor((p[a] - scn->lower[a]) / scn->cell[a]) - off;
        if(g < (int64_t)lo[a]) g = lo[a];
        if(g > (int64_t)hi[a] - 1) g = hi[a] - 1;
        c[a] = (uint32_t)g;
      }
      nc = d[axis] > 0 ? (int64_t)hi[axis] : (int64_t)lo[axis] - 1;
      if(nc < 0 || nc >= (int64_t)scn->def[axis]) {
        if(scn->repeat && axis < 2) {
          if(nc < 0) { tile[axis] -= 1; nc = scn->def[axis] - 1; }
          else { tile[axis] += 1; nc = 0; }
        } else {
          break; /* left the cloud box */
        }
      }
      c[axis] = (uint32_t)nc;
    }
    ta = texit;
  }
  return 0;
}

int
ora_trace_ray(const struct ora_scene* scn, uint32_t band, uint32_t q, int prop,
              const double o[3], const double d[3], const double range[2],
              ora_filter_T filter, void* ctx, struct ora_counters* cnt, struct ora_seg* hit)
{
  double ta = range[0], tb = range[1];
  double cb0, cb1;
  (void)band;
  if(tb > ORA_MAX_DIST) tb = ORA_MAX_DIST;
  slab(o[2], d[2], 0.0, scn->ztop, &ta, &tb);
  if(!(ta < tb)) return 0;
  if(!scn->has_cloud) return trace_gas(scn, q, prop, o, d, ta, tb, filter, ctx, cnt, hit);

  cb0 = ta; cb1 = tb;
  if(!scn->repeat) {
    slab(o[0], d[0], scn->lower[0], scn->upper[0], &cb0, &cb1);
    slab(o[1], d[1], scn->lower[1], scn->upper[1], &cb0, &cb1);
  }
  slab(o[2], d[2], scn->lower[2], scn->upper[2], &cb0, &cb1);
  if(!(cb0 < cb1)) return trace_gas(scn, q, prop, o, d, ta, tb, filter, ctx, cnt, hit);
  if(ta < cb0 && trace_gas(scn, q, prop, o, d, ta, cb0, filter, ctx, cnt, hit)) return 1;
  if(trace_cloud(scn, q, prop, o, d, cb0, cb1, filter, ctx, cnt, hit)) return 1;
  if(cb1 < tb && trace_gas(scn, q, prop, o, d, cb1, tb, filter, ctx, cnt, hit)) return 1;
  return 0;
}

/* Collision site of a point inside a voxel: the cell (clamped to the leaf box)
 * and the gas layer (clamped to the layers the cell overlaps). */
void
ora_site_of(const struct ora_scene* scn, const struct ora_seg* seg, const double p[3],
            struct ora_site* s)
{
  if(!seg->in_cloud) {
    s->cell = -1;
    s->layer = seg->layer;
    return;
  } else {
    uint32_t c[3];
    int a, l;
    for(a = 0; a < 3; ++a) {
      const int64_t off = (a < 2 ? seg->tile[a] * (int64_t)scn->def[a] : 0);
      int64_t g = (int64_t)floor((p[a] - scn->lower[a]) / scn->cell[a]) - off;
      if(g < (int64_t)seg->lo[a]) g = seg->lo[a];
      if(g > (int64_t)seg->hi[a] - 1) g = seg->hi[a] - 1;
      c[a] = (uint32_t)g;
    }
    s->cell = (int64_t)(((size_t)c[2] * scn->def[1] + c[1]) * scn->def[0] + c[0]);
    l = ora_layer_of(scn, p[2]);
    if(scn->cell_layer_lo[c[2]] < 0) l = -1;
    else {
      if(l < scn->cell_layer_lo[c[2]]) l = scn->cell_layer_lo[c[2]];
      if(l > scn->cell_layer_hi[c[2]]) l = scn->cell_layer_hi[c[2]];
    }
    s->layer = l;
  }
}
