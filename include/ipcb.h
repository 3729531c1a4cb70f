/* ipc_warp_b200 C ABI: the per-Newton-iteration IPC contact pipeline on one
 * B200 (sm_100a).
 *
 * Conventions
 *  - Every pointer is a device pointer unless stated otherwise; structs
 *    (ipcb_soup, ipcb_lbvh, ipcb_contacts) are passed by host pointer.
 *  - Positions are AoS scalar[3*V] like the reference's wp.array(dtype=vec3);
 *    `fp64` selects double (the reference's USE_FLOAT32=False build) or float.
 *  - Functions enqueue work on `stream` (a cudaStream_t) and never
 *    synchronize.  They return IPCB_OK or an IPCB_E* code for bad arguments or
 *    a failed launch.  Device-side conditions are reported through device
 *    words the caller reads: contact counts above capacity (overflow: grow
 *    the list and relaunch, as contact.py:523-537,698-723 does) and status
 *    words for bounded loops that ran out (IPCB_STATUS_*).
 *  - Scratch memory is caller-provided: query the size with the *_workspace
 *    function, pass a device block of at least that many bytes.
 */
#ifndef IPCB_H
#define IPCB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* ipcb_stream; /* cudaStream_t */

enum {
  IPCB_OK = 0,
  IPCB_E_ARG = 1,    /* invalid argument (null pointer, negative size, small workspace) */
  IPCB_E_CUDA = 2,   /* a launch or runtime call failed */
};

/* status-word bits written by device code (OR-ed) */
enum {
  IPCB_STATUS_STACK = 1,    /* BVH traversal stack full: result incomplete */
  IPCB_STATUS_ROOT_ITERS = 2, /* cubic root refinement hit its iteration bound */
  IPCB_STATUS_ROW_OVERFLOW = 4, /* contact BSR: a row has more distinct columns than one warp handles */
  IPCB_STATUS_TIMEOUT = 8       /* a bounded wait on the tensor core gave up; outputs are incomplete */
};

/* Geometry: the reference Soup (fem/geometry.py:165-171) plus positions. */
typedef struct {
  int n_verts, n_edges, n_tris;
  int fp64;              /* scalar type of x / xcs: 0 float, 1 double */
  const void* x;         /* scalar[3*n_verts]   soup.x_transformed  */
  const void* xcs;       /* scalar[3*n_verts]   soup.xcs (rest)     */
  const int* edges;      /* int32[2*n_edges]    soup.edges          */
  const int* triangles;  /* int32[3*n_tris]     soup.triangles      */
  const int* body;       /* int32[n_verts]      soup.body           */
} ipcb_soup;

/* Contact list: the reference Contacts/XConstraint (contact.py:61-80) as
 * columns.  Record k: a1a2b1b2[4k..4k+3], e0e1[2k..2k+1], l0[k], alpha[k],
 * lam[k] (scalar = float or double as the soup).  *cnt counts every accepted
 * pair, also those beyond capacity. */
typedef struct {
  int* a1a2b1b2;  /* int32[4*capacity], 16-byte aligned */
  int* e0e1;      /* int32[2*capacity] */
  void* l0;       /* scalar[capacity] */
  void* alpha;    /* scalar[capacity] */
  void* lam;      /* scalar[capacity] */
  int* cnt;       /* int32[1] */
  int capacity;
} ipcb_contacts;

/* Linear BVH over n boxes.  Memory is one caller block carved by
 * ipcb_lbvh_bind.  nodes: 4 float4 per internal node: (L.lo, Lcode),
 * (L.hi, -), (R.lo, Rcode), (R.hi, -); code >= 0 internal node, < 0 leaf
 * ~primitive. */
typedef struct {
  int n;          /* leaves currently built */
  int capacity;   /* leaves the memory was bound for */
  void* nodes;    /* float4[4*max(capacity-1,1)] */
  int* parent;    /* int32[2*capacity]: internal j at j, leaf slot k at capacity+k; (parent<<1)|side, bit 31
                   * set when the parent's leaf range lies in one 32-leaf block */
  int* sorted;    /* int32[capacity]: primitive of each leaf slot (Morton order) */
  unsigned* keys; /* uint32[capacity]: sorted Morton codes */
  unsigned* flags;/* uint32[capacity]: refit arrival counters (zero between calls) */
  void* wide;     /* float4[8*max(capacity-1,1)]: 4-wide view rebuilt by build/refit (queries use it) */
} ipcb_lbvh;

int ipcb_version(void);
/* hash of this header at build time; a loader compares it with its header */
const char* ipcb_abi_hash(void);
const char* ipcb_last_error(void);

/* ---- device radix sort (also used inside build and BSR assembly) ---- */
size_t ipcb_sort_workspace_u32(int n);
size_t ipcb_sort_workspace_u64(int n);
/* Stable sort by the low end_bit bits of keys, values permuted alongside. */
int ipcb_sort_pairs_u32(unsigned* keys, int* vals, int n, int end_bit, void* ws, size_t ws_bytes, ipcb_stream s);
int ipcb_sort_pairs_u64(unsigned long long* keys, int* vals, int n, int end_bit, void* ws, size_t ws_bytes,
                        ipcb_stream s);

/* ---- LBVH (replaces wp.Bvh / wp.Mesh build and .refit(): contact.py:464-483, 672-677) ---- */
size_t ipcb_lbvh_bytes(int capacity);
int ipcb_lbvh_bind(ipcb_lbvh* bvh, void* mem, int capacity);
size_t ipcb_lbvh_build_workspace(int n);
/* 30-bit Morton codes of box centres, radix sort, Karras hierarchy in one
 * kernel, then a bottom-up refit.  lower/upper: float[3n]. */
int ipcb_lbvh_build(ipcb_lbvh* bvh, const float* lower, const float* upper, int n, void* ws, size_t ws_bytes,
                    ipcb_stream s);
/* Recompute node boxes for new leaf boxes, same topology (atomic bottom-up). */
int ipcb_lbvh_refit(const ipcb_lbvh* bvh, const float* lower, const float* upper, ipcb_stream s);

/* LBVH build that allocates nothing.  No counterpart in the reference: it
 * serves callers that cannot call cudaMalloc while a step runs (an allocation
 * may synchronise the device; a host framework may own all device memory in
 * its own pool; a JNI/FFI binding may only pass buffers it already holds).
 * Same result as ipcb_lbvh_build; the build scratch is a file-scope
 * __device__ array of ipcb_lbvh_build_noalloc_scratch_bytes() (about 2.2 MB)
 * that every GPU loading the library keeps until exit, so n is limited to
 * IPCB_LBVH_NOALLOC_MAX_PRIMS (larger n returns IPCB_E_ARG, as does n above the
 * hierarchy's capacity, each with its own ipcb_last_error text).  Every call
 * made outside stream capture looks the array's device address up
 * (cudaGetSymbolAddress) in the context current on the calling thread, so the
 * address stays right after cudaDeviceReset or in a non-primary context; a
 * call inside capture uses the address that the last call outside capture
 * found for that device ordinal, so make one call on each device before
 * capturing, and again after a cudaDeviceReset.  All calls share the one
 * array, so calls that overlap on the GPU race; the build clears what must
 * start at zero, and the array keeps the last call's data. */
#define IPCB_LBVH_NOALLOC_MAX_PRIMS (1 << 18)
size_t ipcb_lbvh_build_noalloc_scratch_bytes(void);
int ipcb_lbvh_build_noalloc(ipcb_lbvh* bvh, const float* lower, const float* upper, int n, ipcb_stream s);

/* ---- boxes (contact.py:30-52, ccd/ccd.py:166-210) ---- */
/* x4 = float4(x) (the reference's float32 mesh copy, contact.py:44-47, as 16-byte records) */
int ipcb_pack_positions(const ipcb_soup* soup, float* x4, ipcb_stream s);
/* edge AABBs of x4 padded by pad (edge_aabb, contact.py:30-37) */
int ipcb_edge_aabbs(const ipcb_soup* soup, const float* x4, float pad, float* lower, float* upper, ipcb_stream s);
/* triangle AABBs of x4 padded by pad (wp.Mesh bounds, contact.py:479,677) */
int ipcb_triangle_aabbs(const ipcb_soup* soup, const float* x4, float pad, float* lower, float* upper,
                        ipcb_stream s);
/* x1 = x - dx in the soup scalar (_add_dx, contact.py:49-52) */
int ipcb_add_dx(const ipcb_soup* soup, const void* dx, void* x1, ipcb_stream s);
/* swept boxes of (x, x1) padded, rounded outward to float (ccd.py:166-210) */
int ipcb_swept_edge_aabbs(const ipcb_soup* soup, const void* x1, double pad, float* lower, float* upper,
                          ipcb_stream s);
int ipcb_swept_triangle_aabbs(const ipcb_soup* soup, const void* x1, double pad, float* lower, float* upper,
                              ipcb_stream s);

/* ---- DCD broad phase (contact.py:199-228 edge_edge_collision, 304-336 point_triangle_collision) ----
 * Appends every pair with float32 closest distance < 2*thickness that passes
 * the reference filters.  The caller zeroes out->cnt first.  query_pad is the
 * query-box inflation (the reference uses thickness+buffer for EE against
 * boxes already inflated by the same, 2*(thickness+buffer) for PT against
 * tight triangle boxes); any pad >= the reference's keeps the candidate set. */
int ipcb_dcd_ee(const ipcb_soup* soup, const float* x4, const ipcb_lbvh* edge_bvh, float thickness, float query_pad,
                int exclude_same_body, ipcb_contacts* out, int* status, ipcb_stream s);
/* query_order: optional int32[n_verts] vertex visiting order (NULL = 0..V-1) */
int ipcb_dcd_pt(const ipcb_soup* soup, const float* x4, const ipcb_lbvh* tri_bvh, float thickness, float query_pad,
                int exclude_same_body, const int* query_order, ipcb_contacts* out, int* status, ipcb_stream s);
/* One scene's queries split over several GPUs: the same queries restricted to
 * the queries first .. first + count - 1 (EE: the edges of those Morton ranks
 * in edge_bvh, and every pair is met by its lower-ranked edge, so disjoint
 * rank ranges partition the pair set; PT: those vertices of the visiting
 * order).  ipcb_dcd_ee / ipcb_dcd_pt are the full ranges. */
int ipcb_dcd_ee_range(const ipcb_soup* soup, const float* x4, const ipcb_lbvh* edge_bvh, float thickness,
                      float query_pad, int exclude_same_body, int first, int count, ipcb_contacts* out, int* status,
                      ipcb_stream s);
int ipcb_dcd_pt_range(const ipcb_soup* soup, const float* x4, const ipcb_lbvh* tri_bvh, float thickness,
                      float query_pad, int exclude_same_body, const int* query_order, int first, int count,
                      ipcb_contacts* out, int* status, ipcb_stream s);

/* ---- narrow phase (dynamic_contacts.py:152-246 contact_hessian_ee/pt, 375-398 energy) ----
 * kind 0 = EE list, 1 = PT list.  n >= 0: number of records; n < 0: read
 * min(*list->cnt, capacity) on the device (graph-capturable).
 * Writes 16 triplets per record at (offset + k)*16 + ii*4 + jj: rows/cols
 * int32, vals scalar[9] row-major; inactive records (dist >= l0) get zero
 * blocks at (0,0).  b (scalar[3V]) accumulates the force -dE/dx.
 * block_mask (optional, uint16[offset + n]): bit ii*4+jj set when block
 * (ii, jj) of the record has a non-zero entry (read by ipcb_contact_bsr). */
int ipcb_contact_hessian(int kind, const ipcb_soup* soup, const ipcb_contacts* list, int n, int offset, double kappa,
                         int* rows, int* cols, void* vals, void* b, unsigned short* block_mask, ipcb_stream s);
/* The same with the record offset taken on the device: records go at
 * (min(*offset_count, offset) + k)*16, so a PT list can follow the EE list's
 * device-side count without a host read (offset = the EE list's capacity). */
int ipcb_contact_hessian_after(int kind, const ipcb_soup* soup, const ipcb_contacts* list, int n, int offset,
                               const int* offset_count, double kappa, int* rows, int* cols, void* vals, void* b,
                               unsigned short* block_mask, ipcb_stream s);
/* ipcb_contact_hessian_after with the list's records first put in cost-class
 * order over the whole list (costliest first: edge-edge / point-triangle
 * eigen-solve, point-edge, no eigen-solve, inactive), so that nearly every
 * warp takes one path through the Hessian: a classification kernel caches
 * each record's float32 distance and feature, a second one writes the order,
 * then the Hessian kernel runs in that order.  Same outputs (each record
 * writes its own slots; only the order of the force atomics differs).
 * ws: ipcb_contact_hessian_workspace(list->capacity) bytes of device memory. */
size_t ipcb_contact_hessian_workspace(int capacity);
int ipcb_contact_hessian_sorted(int kind, const ipcb_soup* soup, const ipcb_contacts* list, int n, int offset,
                                const int* offset_count, double kappa, int* rows, int* cols, void* vals, void* b,
                                unsigned short* block_mask, void* ws, size_t ws_bytes, ipcb_stream s);
/* energy (double) += sum of the barrier energy of the list */
int ipcb_contact_energy(int kind, const ipcb_soup* soup, const ipcb_contacts* list, int n, double kappa,
                        double* energy, ipcb_stream s);

/* ---- intersection check of a surface state ----
 * No single counterpart in the reference: it is the check its trajectories
 * are judged by (an accepted step leaves no surface edge crossing a surface
 * triangle).  Every (edge, triangle) pair without a shared vertex whose
 * segment crosses the triangle's interior (orientation signs in double,
 * touching and coplanar configurations not counted) adds 1 to *count (caller
 * zeroes it); the first `capacity` pairs go to pairs (int32[2*capacity]:
 * edge, triangle).  tri_bvh: the triangle hierarchy refit to soup->x.
 * IPCB_STATUS_STACK in *status when a traversal ran out of its bound. */
int ipcb_edge_triangle_crossings(const ipcb_soup* soup, const ipcb_lbvh* tri_bvh, int* count, int* pairs,
                                 int capacity, int* status, ipcb_stream s);

/* ---- CCD (ccd/ccd.py:360-427 point_triangle_toi / edge_edge_toi) ----
 * Cubic coplanarity TOI in double for every candidate whose swept boxes
 * overlap; toi (scalar[1], caller sets 1) gets the minimum root < 1,
 * rounded toward zero when stored as float.  The workspace stages candidate
 * pairs (ipcb_toi_workspace(capacity) bytes, int32 count first); pairs that
 * do not fit are solved during traversal, so any capacity >= 0 is correct. */
size_t ipcb_toi_workspace(int capacity);
int ipcb_edge_edge_toi(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* swept_edge_bvh, const float* lower,
                       const float* upper, int exclude_same_body, void* toi, int* status, void* ws, size_t ws_bytes,
                       ipcb_stream s);
int ipcb_point_triangle_toi(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* swept_tri_bvh, double pad,
                            int exclude_same_body, void* toi, int* status, void* ws, size_t ws_bytes, ipcb_stream s);
/* The CCD queries restricted to a range of queries, as ipcb_dcd_ee_range /
 * ipcb_dcd_pt_range (EE: Morton ranks of swept_edge_bvh; PT: vertices). */
int ipcb_edge_edge_toi_range(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* swept_edge_bvh,
                             const float* lower, const float* upper, int exclude_same_body, int first, int count,
                             void* toi, int* status, void* ws, size_t ws_bytes, ipcb_stream s);
int ipcb_point_triangle_toi_range(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* swept_tri_bvh, double pad,
                                  int exclude_same_body, int first, int count, void* toi, int* status, void* ws,
                                  size_t ws_bytes, ipcb_stream s);
/* new_intersections (contact.py:587-670; edge_edge_intersections /
 * point_triangle_intersections 371-442): the CCD queries above that also
 * append every pair whose time of impact is < 1 to `out` as a record
 * (append_ccd 186-197: EE a0 a1 b0 b1 with e0e1 = (i, j), i < j; PT the
 * vertex and the triangle's t0 t1 t2 with e0e1 = (vertex, triangle);
 * l0 = 2 thickness, alpha = toi, lam = 0), besides the minimum in toi.
 * *out->cnt counts every such pair; records beyond the capacity are dropped
 * (grow and relaunch, as the reference). */
int ipcb_edge_edge_intersections(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* swept_edge_bvh,
                                 const float* lower, const float* upper, int exclude_same_body, double thickness,
                                 void* toi, const ipcb_contacts* out, int* status, void* ws, size_t ws_bytes,
                                 ipcb_stream s);
int ipcb_point_triangle_intersections(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* swept_tri_bvh,
                                      double pad, int exclude_same_body, double thickness, void* toi,
                                      const ipcb_contacts* out, int* status, void* ws, size_t ws_bytes,
                                      ipcb_stream s);
/* per-pair collision time of n explicit pairs (kind 0 EE, 1 PT); p_t0/p_t1:
 * double[n*12] (4 points each) -> t double[n] (ee/pt_collision_time, ccd.py:304-357) */
int ipcb_collision_time(int kind, int n, const double* p_t0, const double* p_t1, double* t, int* status,
                        ipcb_stream s);
/* cubic_roots (cubic_roots.py:96-193) of n cubics coef double[4n] on [x0,x1] */
int ipcb_cubic_roots(int n, const double* coef, double x0, double x1, double* roots, int* n_roots, int* status,
                     ipcb_stream s);

/* ---- FEM elastic term (fem/fem.py:22-34 compute_Dm, 139-203 tet_kernel_sparse;
 *      time_integrator_base.py:124-137 compute_Psi) ----
 * material: 0 stable Neo-Hookean (fem/snh.py), 1 Neo-Hookean (fem/neo_hookean.py),
 * 2 St. Venant-Kirchhoff (fem/stvk.py); Lame mu, lam.  tets int32[4n].
 * rest: Bm = Dm^-1 (scalar[9n] row-major), W = |det Dm|/6.
 * hessian: 16 triplets per tet at tet*16 + i*4 + j (K_ij, not projected,
 * as the reference; rows and cols may both be null when the caller keeps the
 * pattern) and the nodal forces added to b.  energy += sum W psi(F). */
int ipcb_tet_rest(int fp64, const void* xcs, const int* tets, int n_tets, void* Bm, void* W, ipcb_stream s);
int ipcb_tet_hessian(int material, int fp64, const void* x, const int* tets, int n_tets, const void* Bm, const void* W,
                     double mu, double lam, int* rows, int* cols, void* vals, void* b, ipcb_stream s);
int ipcb_tet_energy(int material, int fp64, const void* x, const int* tets, int n_tets, const void* Bm, const void* W,
                    double mu, double lam, double* energy, ipcb_stream s);

/* ---- Body-local (fixed) hierarchies for affine bodies ----
 * fixed_bvh_contacts.py:32-827 (FixedBodyContactSolver): every body keeps the
 * hierarchies of its rest-frame edges and triangles, built once; a query
 * primitive of body a is mapped into body b's rest frame (x_local =
 * A_b^-1 (x - p_b)) and tested against b's hierarchy, then accepted by the
 * same exact world-space predicate and append as ipcb_dcd_ee / ipcb_dcd_pt.
 * q: scalar[12 nb], per body p, A[:,0], A[:,1], A[:,2] (x = p + A r,
 * affine_body_dynamics.py:1-10).  Per-body primitive lists: the primitives of
 * body b are ids[off[b] .. off[b+1]); the 4-wide hierarchy of body b
 * (ipcb_lbvh.wide of a tree built over its rest boxes in that order) is
 * edge_wide[b] / tri_wide[b].  frames: double[19 nb] scratch (A^-1, p,
 * |A^-1|_F, then the world boxes), motion: double[3 nb] scratch, written by
 * the pair culls; int32 grids cap pairs x chunks at 2^31 blocks. */
#define IPCB_STATUS_SINGULAR 32 /* a body's |det A| < 1e-8: use the dynamic path */

typedef struct {
  int n_bodies;
  const float* local_lower;
  const float* local_upper;
  const int* edge_off;
  const int* edge_ids;
  const int* tri_off;
  const int* tri_ids;
  const int* vert_off;
  const int* vert_ids;
  const void* const* edge_wide;
  const void* const* tri_wide;
  int max_edges, max_tris, max_verts;
  double* frames;
  double* motion;
} ipcb_bodies;

/* Overlapping body pairs (a < b) of the world boxes of the affine bodies,
 * padded by `padding` (affine_body_aabbs + compact_overlapping_body_pairs,
 * fixed_bvh_contacts.py:48-99); also fills `frames`.  pairs int2[capacity],
 * *count may exceed capacity (grow and relaunch). */
int ipcb_body_pairs(const ipcb_bodies* B, int fp64, const void* q, double padding, int* pairs, int capacity,
                    int* count, int* status, ipcb_stream s);
/* EE (source body = pair.x) and PT (both directions) queries of
 * batched_fixed_bvh_edge_edge_query / _point_triangle_query
 * (fixed_bvh_contacts.py:295-380): padding |A^-1|_F * 2 thickness. */
int ipcb_fixed_dcd_ee(const ipcb_soup* soup, const float* x4, const ipcb_bodies* B, const int* pairs, int n_pairs,
                      float thickness, ipcb_contacts* out, int* status, ipcb_stream s);
int ipcb_fixed_dcd_pt(const ipcb_soup* soup, const float* x4, const ipcb_bodies* B, const int* pairs, int n_pairs,
                      float thickness, ipcb_contacts* out, int* status, ipcb_stream s);
/* Swept body pairs for the step x -= dq (affine_swept_body_aabbs,
 * fixed_bvh_contacts.py:144-175): boxes of the bodies at q and q - dq, also
 * `frames` (at q) and `motion` (the target-frame motion extent,
 * _target_motion_extent 121-141); IPCB_STATUS_SINGULAR when a body's
 * |det A| < 1e-8 at either end. */
int ipcb_body_pairs_swept(const ipcb_bodies* B, int fp64, const void* q, const void* dq, double padding, int* pairs,
                          int capacity, int* count, int* status, ipcb_stream s);
/* CCD over the fixed hierarchies (batched_fixed_bvh_edge_edge_toi /
 * _point_triangle_toi, fixed_bvh_contacts.py:178-292): swept local query
 * boxes inflated by the target's motion extent and |A^-1|_F * pad; the TOI
 * of each candidate is the same exact computation as ipcb_edge_edge_toi.
 * fixed: int32[nb] fixed-body flags (an EE query runs from the moving body). */
int ipcb_fixed_edge_edge_toi(const ipcb_soup* soup, const void* x1, const ipcb_bodies* B, const int* fixed,
                             const int* pairs, int n_pairs, double pad, void* toi, int* status, void* ws,
                             size_t ws_bytes, ipcb_stream s);
int ipcb_fixed_point_triangle_toi(const ipcb_soup* soup, const void* x1, const ipcb_bodies* B, const int* pairs,
                                  int n_pairs, double pad, void* toi, int* status, void* ws, size_t ws_bytes,
                                  ipcb_stream s);

/* ---- Affine body dynamics (affine_body_dynamics.py:33-217, 427-505) ----
 * State of nb affine bodies, every array scalar (fp64 ? double : float):
 * q, q0, q_tilde, qdot, dx: [12 nb], per body p, a0, a1, a2 (ABDState, 33-39;
 * x = p + r0 a0 + r1 a1 + r2 a2); mass: [16 nb] scalar moments M_ij of
 * _build_mass_blocks (344-358, which stores M_ij * I); volume, stiffness:
 * [nb]; fixed: int32[nb]. */
typedef struct {
  int n_bodies;
  int fp64;
  void* q;
  void* q0;
  void* q_tilde;
  void* qdot;
  void* dx;
  const void* mass;
  const void* volume;
  const void* stiffness;
  const int* fixed;
} ipcb_abd;
#define IPCB_ABD_MAX_BODIES 16384 /* reduced-pattern bitmap limit */

/* out[v] = q[b] + r0 q[b+1] + r1 q[b+2] + r2 q[b+3] with b = 4 body[v]:
 * _sync_affine_vertices (42-48) with q, _affine_vertex_direction (51-57) with dx. */
int ipcb_abd_map(int fp64, int n_verts, const void* q, const void* rest, const int* body, void* out, ipcb_stream s);
/* q = q_start - alpha dq (the copy + _affine_add_step of line_search, 60-63, 623-627) */
int ipcb_abd_step_from(int fp64, int n, const void* q_start, const void* dq, double alpha, void* q, ipcb_stream s);
/* _prepare_tilde (66-79); gravity: host double[3]; motor_omega scalar[3 nb]
 * and motor_enabled int32[nb] may be null (no motors). */
int ipcb_abd_prepare_tilde(const ipcb_abd* abd, double h, const double* gravity, const void* motor_omega,
                           const int* motor_enabled, ipcb_stream s);
/* _update_affine_velocity (82-86): qdot = (q - q0) / h, q0 = q */
int ipcb_abd_update_velocity(const ipcb_abd* abd, double h, ipcb_stream s);
/* _assemble_body_system (88-141) in the reference layout: 16 triplets per
 * body at b*16 + i*4 + j (rows/cols int32, vals scalar[9]) and the body
 * gradient rows [4 nb][3]. */
int ipcb_abd_body_system(const ipcb_abd* abd, double h2, int* rows, int* cols, void* vals, void* gradient,
                         ipcb_stream s);
/* _body_energy (193-217): energies[0] += inertia, energies[1] += orthogonality (double) */
int ipcb_abd_body_energy(const ipcb_abd* abd, double h2, double* energies, ipcb_stream s);
/* _reduce_contact_force (144-157): reduced_force[4 nb][3] += J^T f (bodies not fixed) */
int ipcb_abd_reduce_force(const ipcb_abd* abd, int n_verts, const void* vertex_force, const void* rest,
                          const int* body, void* reduced_force, ipcb_stream s);
/* _add_contact_gradient (160-163): gradient -= h2 * force, n scalars */
int ipcb_abd_add_contact_gradient(int fp64, int n, void* gradient, const void* force, double h2, ipcb_stream s);
/* _reduce_contact_hessian (166-190): 16 triplets per source block at
 * src*16 + a*4 + c, zero when either body is fixed. */
int ipcb_abd_reduce_hessian(const ipcb_abd* abd, int n_src, const int* src_rows, const int* src_cols,
                            const void* src_vals, const void* rest, const int* body, double scale, int* dst_rows,
                            int* dst_cols, void* dst_vals, ipcb_stream s);
/* Block pattern of the reduced matrix without the 16x fan-out: every body's
 * diagonal 4x4 block plus the 4x4 blocks of each body pair joined by a
 * contact record (records as ipcb_contact_hessian writes them, 16 triplets
 * each; block_mask optional; pairs with a fixed body are left out).
 * body_off int32[nb+1], body_cols int32[pair_capacity] (the sorted body
 * neighbours, diagonal included), offsets int32[4 nb + 1], columns
 * int32[16 pair_capacity]; *nnz (device) = 16 * body_off[nb].
 * IPCB_STATUS_PATTERN when body_off[nb] > pair_capacity (grow, rerun) or a
 * record spans more than two bodies.  ws: ipcb_abd_pattern_workspace bytes. */
size_t ipcb_abd_pattern_workspace(int n_bodies);
int ipcb_abd_pattern(int n_bodies, const int* fixed, const int* body, int n_records, const int* trows,
                     const int* tcols, const unsigned short* block_mask, int* body_off, int* body_cols,
                     int pair_capacity, int* offsets, int* columns, int* nnz, int* status, void* ws, size_t ws_bytes,
                     ipcb_stream s);
/* The reduced Newton system of AffineBodyDynamics.compute_A (427-505) into
 * the pattern of ipcb_abd_pattern: values (capacity blocks) = body blocks +
 * h2 * J^T H_contact J, gradient [4 nb][3] = body gradient - h2 * J^T f.
 * Records [0, n_ee) are EE records (a1 a2 on one body, b1 b2 on one body),
 * the rest PT (the point on one body, the triangle on one body).
 * vertex_force (scalar[3 n_verts], may be null) with reduced_force
 * (scalar[12 nb], overwritten with J^T f). */
int ipcb_abd_assemble(const ipcb_abd* abd, double h2, int n_records, int n_ee, const int* trows, const int* tcols,
                      const void* tvals, const unsigned short* block_mask, const void* rest, const int* body,
                      const int* body_off, const int* body_cols, const int* offsets, const int* nnz, int capacity,
                      void* values, void* gradient, int n_verts, const void* vertex_force, void* reduced_force,
                      int* status, ipcb_stream s);

/* ---- Mixed FEM + affine-body systems (one Newton solve over tets and affine bodies) ----
 * Unknowns q: n_fem FEM vertex positions, then p, a0, a1, a2 per affine body
 * (the q layout of affine_body_dynamics.py:42-48).  Soup vertex v < n_fem is
 * unknown v; vertex v >= n_fem belongs to body[v - n_fem] with body-local
 * rest position rest[v] (x = p + A r); fixed bodies (fixed[b] != 0) have no
 * unknowns.  rest: scalar[3 n_verts] (the soup's xcs). */
typedef struct {
  int fp64;
  int n_fem;
  int n_verts;
  int n_bodies;
  const int* body;  /* int32[n_verts - n_fem] */
  const int* fixed; /* int32[n_bodies] */
  const void* rest; /* scalar[3 n_verts] */
} ipcb_mixed;
/* x[v] = J_v q: the unknown itself (FEM) or the affine map (_sync_affine_vertices
 * 42-48 on the body part); also maps a direction dq to the vertex direction. */
int ipcb_mixed_map(const ipcb_mixed* m, const void* q, void* x, ipcb_stream s);
/* gradient[unknowns] += scale J^T f (f: scalar[3 n_verts]); fixed bodies get nothing. */
int ipcb_mixed_reduce_force(const ipcb_mixed* m, const void* vertex_force, double scale, void* gradient,
                            ipcb_stream s);
/* Contact Hessian triplets (16 per record, block_mask may be null) -> the
 * unknown-space triplets of J^T H J times scale, written compactly; *n_out
 * (device) = their count; IPCB_STATUS_PATTERN in *status when it exceeds
 * capacity (grow to *n_out and rerun).  ws: ipcb_mixed_hessian_workspace bytes. */
size_t ipcb_mixed_hessian_workspace(int n_src);
int ipcb_mixed_reduce_hessian(const ipcb_mixed* m, int n_src, const int* rows, const int* cols, const void* vals,
                              const unsigned short* block_mask, double scale, int capacity, int* drows, int* dcols,
                              void* dvals, int* n_out, int* status, void* ws, size_t ws_bytes, ipcb_stream s);
/* Pins (pendulum rods): body b's local point pin_rest[b] held at world point
 * pin_target[b] by the energy 0.5 h2 pin_k[b] |x_pin - target|^2 (pin_k 0: no
 * pin).  Optional outputs: 16 triplets per body (rows/cols/vals, all or none),
 * gradient += (unknown layout), *energy += (double). */
int ipcb_mixed_pins(const ipcb_mixed* m, const void* q, const void* pin_rest, const void* pin_target,
                    const void* pin_k, double h2, int* rows, int* cols, void* vals, void* gradient, double* energy,
                    ipcb_stream s);

/* ---- Batched Newton terms and fixed-pattern assembly (time_integrator_base.py:403-426,
 * dynamic_contacts.py:275-297, fem/fem.py:139-203, affine_body_dynamics.py:88-141) ----
 * One persistent launch over all per-iteration terms: the EE records, the PT
 * records (counts read on the device: min(*cnt, capacity)), the tets and the
 * affine bodies' 16 (i, j) items, in that order, with the outputs of
 * ipcb_contact_hessian_sorted (EE at 0, PT at offset n_ee; ee_ws / pt_ws are
 * each list's ipcb_contact_hessian_workspace, the call runs the two ordering
 * passes first), ipcb_tet_hessian (t_rows/t_cols may be null) and
 * ipcb_abd_body_system (triplets a_rows/a_cols/a_vals, 16 per body, at rows
 * body_row0 + 4 b + i; gradient rows written into a_grad; abd.n_bodies may
 * be 0); forces add into `force`.  Work is taken from *queue (zeroed by the
 * call) in tiles of `tile` items per warp (a multiple of 32); blocks x
 * threads (<= 128, multiple of 32) is the persistent grid, with 145 * 32
 * scalars of shared memory per warp. */
typedef struct {
  int fp64;
  const void* x;
  const void* xcs;
  ipcb_contacts ee;
  ipcb_contacts pt;
  double kappa;
  int* c_rows;
  int* c_cols;
  void* c_vals;
  unsigned short* c_mask;
  int material;
  const int* tets;
  int n_tets;
  const void* Bm;
  const void* W;
  double mu, lam;
  int* t_rows;
  int* t_cols;
  void* t_vals;
  void* force;
  int* queue;
  void* ee_ws;
  void* pt_ws;
  ipcb_abd abd;
  int body_row0;
  double h2;
  int* a_rows;
  int* a_cols;
  void* a_vals;
  void* a_grad;
} ipcb_terms;
/* variant 0: the kernel's register budget allows 3 CTAs of 128 per SM; 1: 2 CTAs (255 registers) */
int ipcb_terms_launch(const ipcb_terms* terms, int blocks, int threads, int tile, int variant, ipcb_stream s);
/* slots[i] = position of block (rows[i], cols[i]) in a BSR pattern, -1 if absent */
int ipcb_bsr_slots(int nrow, const int* offsets, const int* columns, int n, const int* rows, const int* cols,
                   int* slots, ipcb_stream s);
/* Union of two BSR patterns with the same rows: c_off[nrow+1], and per slot
 * c_rows, c_cols, src_a / src_b (the slot in a / b, -1 if absent); *c_nnz
 * (device).  IPCB_STATUS_PATTERN when the union exceeds capacity. */
size_t ipcb_bsr_union_workspace(int nrow);
int ipcb_bsr_union(int nrow, const int* a_off, const int* a_cols, const int* b_off, const int* b_cols, int* c_off,
                   int* c_rows, int* c_cols, int* src_a, int* src_b, int capacity, int* c_nnz, int* status, void* ws,
                   size_t ws_bytes, ipcb_stream s);
/* Values of the union: slot p = tet_scale * sum of the tet blocks gathered
 * through gather_off/gather_idx (a CSR from each slot of pattern a to the
 * triplets landing on it) + diag[row] I on the diagonal (diag may be null)
 * + contact_scale * contact_vals[src_b[p]]. */
int ipcb_newton_values(int fp64, const int* nnz, int capacity, const int* c_rows, const int* c_cols, const int* src_a,
                       const int* src_b, const int* gather_off, const int* gather_idx, const void* tet_vals,
                       double tet_scale, const void* diag, const void* contact_vals, double contact_scale,
                       void* values, ipcb_stream s);

/* ---- Device-side line search (time_integrator_base.py:514-546) ----
 * State of one backtracking search in device memory.  ipcb_ls_begin: E0 from
 * the energy accumulators acc[3] (acc[0] elastic Psi, acc[1] barrier, acc[2]
 * inertia + attachment; E = h2 (acc0 + acc1) + acc2), the bound from the CCD
 * toi (0.9 toi if toi < 1, else 1).  status (may be null) is the CCD queries'
 * status word: with IPCB_STATUS_STACK or IPCB_STATUS_ROOT_ITERS set the TOI
 * is no bound, so the search is refused (refused = the bits, bound 0, one
 * trial at alpha 0, nothing accepted).  Per trial: ipcb_ls_trial (x = x_tmp -
 * alpha dx, acc zeroed), the energy kernels, ipcb_ls_accept (accept if E1
 * finite and < E0, else halve alpha; stops at alpha <= eps max(1, ub), at
 * max_it trials or when a contact list count exceeds its capacity; sets the
 * WHILE condition of cond_handle when non-zero).  ipcb_ls_finish restores x
 * when nothing was accepted. */
typedef struct {
  double E0, E1, alpha, ub, eps, alpha_accepted;
  int it, max_it, accepted, done, overflow, max_ee, max_pt, refused;
} ipcb_ls_state;
/* acc += inertia 1/2 m |x - x~|^2 (x~ = x0 + h xdot + h^2 g) + attachment
 * 1/2 k_att h^2 |x - target|^2 over fixed vertices, in double; fixed: uint8[V]
 * or null; gravity: host double[3]. */
int ipcb_ls_inertia(int fp64, int n, const void* x, const void* x0, const void* xdot, const double* gravity, double h,
                    const double* mass, const unsigned char* fixed, const void* target, double k_att, double* out,
                    ipcb_stream s);
int ipcb_ls_begin(ipcb_ls_state* st, const void* toi, int fp64, const int* status, const double* acc, double h2,
                  double eps, int max_it, const ipcb_contacts* ee, const ipcb_contacts* pt, ipcb_stream s);
int ipcb_ls_trial(const ipcb_ls_state* st, int fp64, int n_verts, const void* x_tmp, const void* dx, void* x,
                  double* acc, ipcb_stream s);
int ipcb_ls_accept(ipcb_ls_state* st, const double* acc, double h2, const ipcb_contacts* ee, const ipcb_contacts* pt,
                   unsigned long long cond_handle, ipcb_stream s);
int ipcb_ls_finish(const ipcb_ls_state* st, int fp64, int n_verts, const void* x_tmp, void* x, ipcb_stream s);
/* *acc += extra[0] + ... + extra[n-1], then extra[0 .. n) = 0 (one thread, in
 * this order): folds energy terms accumulated apart (affine-body inertia and
 * orthogonality, pins, FEM inertia) into the inertia slot of a line-search
 * accumulator without a host read. */
int ipcb_acc_fold(double* acc, double* extra, int n, ipcb_stream s);
/* A CUDA graph with one WHILE conditional node: _begin creates it and starts
 * capturing stream s (not the legacy default stream) into the loop body
 * (*handle: the condition, 1 at the start of every launch); launches on s
 * until _end form the body; _launch runs the loop; _destroy frees it. */
int ipcb_graph_while_begin(void** ctx, unsigned long long* handle, ipcb_stream s);
int ipcb_graph_while_end(void* ctx, ipcb_stream s);
int ipcb_graph_launch(void* ctx, ipcb_stream s);
void ipcb_graph_destroy(void* ctx);

/* ---- Hashed active set of the augmented-Lagrangian solver
 * (augmented_lagrangian.py:105-198 kernels, 506-572 ActiveSet) ----
 * ALConstraint columns (capacity entries, scalar = fp64 ? double : float)
 * stored bucket by bucket; bucket b of the key e0e1 (hash_pos: (e0 * 73856093
 * xor e1 * 19349663) in 32-bit, non-negative, mod table_size) holds entries
 * cell_start[b] .. cell_start[b+1]; cell_start[table_size] = count. */
typedef struct {
  int table_size;
  int capacity;
  int* cell_start;   /* int32[table_size + 1] */
  int* a1a2b1b2;     /* int4[capacity] */
  int* e0e1;         /* int2[capacity] */
  void* l0;
  void* alpha;
  void* lam;
  void* gamma;
  void* slack;
  void* mollifier;
  void* d0;
  int* distance_type;
  void* grad;        /* scalar[12 capacity] */
} ipcb_al_set;
/* accumulate_vertex_toi: vertex_toi[v] = min(vertex_toi[v], alpha) over the
 * n records' vertices (vertex_toi scalar[V], non-negative on entry) */
int ipcb_al_vertex_toi(int fp64, const ipcb_contacts* list, int n, void* vertex_toi, ipcb_stream s);
size_t ipcb_al_workspace(int table_size);
/* ActiveSet.create_hash: the records kept by filter_accept (alpha <= the
 * toi of one of its vertices + 1e-12), as fresh constraints (lam 0, gamma 1,
 * slack 0, mollifier 1, type 0, d0 0, grad 0); n <= set->capacity. */
int ipcb_al_create(int fp64, ipcb_al_set* set, const ipcb_contacts* list, int n, const void* vertex_toi, void* ws,
                   size_t ws_bytes, ipcb_stream s);
/* ActiveSet.merge: dst = the old entries with gamma >= 0.01 and the new
 * entries whose key is not in old; n_new + n_old <= dst->capacity. */
int ipcb_al_merge(int fp64, const ipcb_al_set* nw, const ipcb_al_set* old, ipcb_al_set* dst, int n_new, int n_old,
                  void* ws, size_t ws_bytes, ipcb_stream s);

/* ---- BSR assembly (warp.sparse.bsr_from_triplets, dynamic_contacts.py:290-297) ----
 * Canonical 3x3-block CSR from triplets: sort by (row, col), sum duplicates,
 * drop triplets whose 9 values are all zero.  offsets int32[nrow+1],
 * columns int32[>= n_trip], values scalar[9*n_trip]; *nnz gets the block count. */
size_t ipcb_bsr_workspace(int n_trip, int nrow, int ncol);
int ipcb_bsr_from_triplets(int nrow, int ncol, int n_trip, const int* rows, const int* cols, const void* vals,
                           int fp64, int* offsets, int* columns, void* values, int* nnz, void* ws, size_t ws_bytes,
                           ipcb_stream s);
/* The same BSR for the contact Hessian, assembled from the EE and PT lists,
 * their triplet values (16 blocks per record, EE records first, as
 * ipcb_contact_hessian writes them) and block masks instead of from generic
 * triplets: the
 * records' structure (one row and 4 columns per (record, slot)) replaces the
 * per-triplet bucketing.  Deterministic.  If a row has more than 128 distinct
 * columns, *status gets IPCB_STATUS_ROW_OVERFLOW and the caller must use
 * ipcb_bsr_from_triplets instead.  n_ee < 0 (n_pt < 0): that list's count is
 * min(*cnt, capacity), read on the device (the PT records then follow that
 * many EE records, as ipcb_contact_hessian_after writes them); the
 * workspace and the capacity of columns/values are sized for the
 * capacities. */
size_t ipcb_contact_bsr_workspace(int n_records, int n_verts);
int ipcb_contact_bsr(const ipcb_contacts* ee, int n_ee, const ipcb_contacts* pt, int n_pt, int n_verts,
                     const void* vals, const unsigned short* block_mask, int fp64, int* offsets, int* columns,
                     void* values, int* nnz, int* status, void* ws, size_t ws_bytes, ipcb_stream s);
/* y = alpha*A*x + beta*y for a 3x3 BSR (bsr_mv) */
int ipcb_bsr_mv(int nrow, const int* offsets, const int* columns, const void* values, int fp64, const void* x,
                void* y, double alpha, double beta, ipcb_stream s);

/* ---- Learned preconditioner: message-passing net -> FSAI factor ----
 * No counterpart in the reference (its linear solve is cg or cuDSS LDLT,
 * time_integrator_base.py:470-507).  A 4-layer, width-64 message-passing net
 * over the 3x3-block graph of a Newton matrix A (canonical BSR: sorted,
 * structurally symmetric, every diagonal block present) predicts the row
 * directions H of a block lower-triangular factor on the lower pattern of A;
 * ipcb_fsai_normalize scales each block row exactly (G^_i = C_i^-1 H_i with
 * C_i C_i^T = M_i = H_i A^ H_i^T, A^ = S A S, S = diag(A)^-1/2 per scalar), so
 * every diagonal block of G^ A^ G^T is I, and M^-1 = S G^T G^ S
 * preconditions PCG.  The training loss is (1/N) sum_i log det M_i (the
 * Kaporin condition number of the normalised factor, up to a constant).
 * Products run on the tensor cores (BF16 operands, FP32 accumulation); H, G^
 * and everything the solve touches are FP32.
 *
 * Graph arrays (device, int32): rows[nnz] (row of each block), rev[nnz]
 * (index of the transposed block), diag[n] (index of (i, i)), lower[n_lower]
 * (blocks with column <= row, in block order; n_lower = (nnz + n) / 2). */
#define IPCB_MPNN_WIDTH 64
#define IPCB_MPNN_IN 16
#define IPCB_MPNN_LAYERS 4
#define IPCB_STATUS_PATTERN 16 /* pattern not symmetric / diagonal missing / non-positive diagonal */

typedef struct {
  int n, nnz, n_lower;
  const int* offsets; /* int32[n + 1] */
  const int* columns; /* int32[nnz] */
  int* rows;
  int* rev;
  int* diag;
  int* lower;
} ipcb_graph;

/* Parameter layout: FP32 master vector (weights stored in x out, row-major,
 * then the bias, per linear map: W_hin b_hin W_ein b_ein, per layer
 * W1 b1 W2 b2, then the head W_off b_off) and the BF16 operand copies the
 * kernels read (made by ipcb_mpnn_pack). */
int ipcb_mpnn_param_count(void);
int ipcb_mpnn_packed_count(void);
int ipcb_mpnn_pack(const float* params, void* packed, ipcb_stream s);

size_t ipcb_mpnn_graph_workspace(int n);
int ipcb_mpnn_graph(ipcb_graph* g, int* status, void* ws, size_t ws_bytes, ipcb_stream s);
/* Scaling s (float[3n]), scaled blocks ahat (float[9 nnz]) and the net's
 * inputs x (bf16[16 n]) and y (bf16[16 nnz]) from the BSR values. */
int ipcb_mpnn_features(const ipcb_graph* g, int fp64, const void* values, float* scale, float* ahat, void* x,
                       void* y, int* status, ipcb_stream s);

/* Activations: bf16 buffers; h[5][n*64], e[5][nnz*64] (layer inputs and the
 * final state), m[4][nnz*64], a[4][n*64], u[4][n*64]; for inference only
 * h[0..1], e[0..1] (ping-pong), m[0] and a[0] are used and u may be NULL.
 * proj: float[n*128] scratch. */
typedef struct {
  void* h;
  void* e;
  void* m;
  void* a;
  void* u;
  float* proj;
  int training;
} ipcb_mpnn_tape;

/* H: float[9 nnz], written on the lower blocks: H_ii = I and
 * H_ij = (rho_i out - I) A^_ij, with out the head output read as a 3x3
 * matrix and rho_i = c / (1 + c) (c: the row's summed |A^_ij|_F, node
 * feature 10); a zero head gives first-order FSAI (ahat, x from
 * ipcb_mpnn_features). */
int ipcb_mpnn_forward(const ipcb_graph* g, const void* packed, const float* params, const float* ahat, const void* x,
                      const void* y, ipcb_mpnn_tape* tape, float* H, int* status, ipcb_stream s);
/* G^ (float[9 nnz], lower blocks) from H: T (float[9 nnz] scratch) gets
 * T_ij = sum_k H_ik A^_kj, minv (float[9 n]) gets M_i^-1, acc[0] (double,
 * device) += sum_i log det M_i.  A row whose M_i is not positive definite
 * keeps G^ = H and raises IPCB_STATUS_PATTERN. */
int ipcb_fsai_normalize(const ipcb_graph* g, const float* ahat, const float* H, float* T, float* minv, float* G,
                        double* acc, int* status, ipcb_stream s);
/* Gradient of weight * (1/N) sum_i log det M_i w.r.t. the head outputs,
 * after ipcb_fsai_normalize: dG bf16[64 n_lower], columns 0..8 (zero rows for
 * diagonal blocks). */
int ipcb_mpnn_loss_grad(const ipcb_graph* g, const float* ahat, const void* x, const float* T, const float* minv,
                        void* dG, double weight, ipcb_stream s);
size_t ipcb_mpnn_backward_workspace(int n, int nnz, int n_lower);
/* Gradients of sum(dG * head outputs) w.r.t. the parameters, added to grad
 * (float[param_count]).  Needs the training tape of the forward call. */
int ipcb_mpnn_backward(const ipcb_graph* g, const void* packed, const float* params, const void* x, const void* y,
                       const ipcb_mpnn_tape* tape, const void* dG, float* grad, int* status, void* ws,
                       size_t ws_bytes, ipcb_stream s);
/* One Adam step (bias-corrected, step t >= 1) over n parameters. */
int ipcb_adam(int n, float* params, const float* grad, float* m, float* v, float lr, float beta1, float beta2,
              float eps, int t, ipcb_stream s);
/* z = S G^T G^ S r (r, z: scalar[3n]; fp64 selects double vectors); tmp:
 * float/double[3n]. */
int ipcb_fsai_apply(const ipcb_graph* g, const float* G, const float* scale, int fp64, const void* r, void* tmp,
                    void* z, ipcb_stream s);

/* ---- Device-resident PCG (time_integrator_base.py:502-507, ``cg``) ----
 * Solves A x = b on the canonical BSR with x0 = 0 to |r| <= tol |b|; the
 * scalars live in `state` (device), so batches of iterations run without a
 * host synchronisation (and can be replayed as a CUDA graph); a finished
 * solve turns further launches into no-ops.  precond 0: block Jacobi (dinv:
 * inverse diagonal blocks, scalar[9n], from ipcb_block_jacobi); precond 1:
 * the learned FSAI factor (diag: int32[n] diagonal block indices, g: bf16
 * [9 nnz] from ipcb_fsai_mirror on its own pattern g_offsets / g_columns,
 * scale: float[3n], t: scalar[3n] scratch).  The factor's pattern may differ
 * from A's (a factor kept from an earlier Newton matrix is still an SPD
 * preconditioner).  state->status bit 1: breakdown (p.Ap <= 0). */
typedef struct {
  double rz, rz_new, pAp, rr, bb, tol2, last_rr;
  int it, done, maxiter, status;
  int arrived; /* blocks of the last kernel of an iteration that have finished (internal) */
} ipcb_pcg_state;

typedef struct {
  int n, fp64, precond;
  const int* offsets;
  const int* columns;
  const void* values;
  const void* dinv;
  const int* g_offsets;
  const int* g_columns;
  const int* diag;
  const void* g;
  const float* scale;
  const void* b;
  void *x, *r, *z, *p, *q, *t;
  ipcb_pcg_state* state;
  /* precond 0 with n_groups > 0 (a mixed FEM + affine-body system): rows
   * n_point + 4 g .. + 3 form group g (one affine body's p, a0, a1, a2) and
   * use the inverse of their 12x12 diagonal block, dinv_group scalar[144
   * n_groups] from ipcb_group_jacobi; n = n_point + 4 n_groups. */
  int n_point, n_groups;
  const void* dinv_group;
  /* initial guess scalar[3n], or NULL for x = 0: ipcb_pcg_start copies it to
   * x and starts from r = b - A x0 (the stopping test stays relative to |b|) */
  const void* x0;
} ipcb_pcg;

int ipcb_pcg_start(const ipcb_pcg* P, double tol, int maxiter, ipcb_stream s);
int ipcb_pcg_iterate(const ipcb_pcg* P, int k, ipcb_stream s);
/* Inverse diagonal blocks (diag may be NULL: found by a row scan). */
int ipcb_block_jacobi(int n, const int* offsets, const int* columns, const int* diag, const void* values, int fp64,
                      void* dinv, int* status, ipcb_stream s);
/* Inverses of the 12x12 diagonal blocks of the row groups n_point + 4 g .. + 3
 * (g < n_groups), row-major scalar[144 n_groups]; IPCB_STATUS_PATTERN when a
 * block is singular (its inverse is then the identity). */
int ipcb_group_jacobi(int n_point, int n_groups, const int* offsets, const int* columns, const void* values,
                      int fp64, void* dinv_group, int* status, ipcb_stream s);
/* bf16 copy of the FSAI factor for the apply: lower and diagonal blocks as
 * they are, upper slots holding the transposed lower block. */
int ipcb_fsai_mirror(const ipcb_graph* g, const float* G, void* gh, ipcb_stream s);

/* ---- BF16 tensor-core GEMM (tcgen05, TMEM accumulator) ----
 * No counterpart in the reference: the building block of the learned
 * preconditioner's kernels, exported for its own tests and for callers that
 * need a plain GEMM.  C[M x N] (fp32) = A[M x K] * B[N x K]^T, A and B
 * row-major bf16; N in {16, 64, 128, 192, 256}, K in {64, 128, 192, 256}.
 * *status gets IPCB_STATUS_TIMEOUT if a bounded wait gave up. */
int ipcb_umma_gemm_bf16(int M, int N, int K, const void* A, const void* B, void* C, int* status, ipcb_stream s);

#ifdef __cplusplus
}
#endif
#endif /* IPCB_H */
