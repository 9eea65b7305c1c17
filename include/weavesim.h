/* weavesim.h — C ABI of the B200 dynamic-relaxation solver for woven (Kagome) timber gridshells.
 *
 * Drop-in boundary for the solver API of weave-sim's web/js solvers:
 *   scene (laths, crossings, supports, material) -> relax -> node positions, segment frames, crossing slide
 *   coordinates and stick/slip states.
 * Every entry point is extern "C", takes plain pointers and sizes, never throws, and returns an int status
 * (WS_OK = 0, < 0 on error; ws_last_error() gives the message of the last failure on the calling thread).
 * Citations are file:line in the reference project (uwenji/weave-sim).
 */
#ifndef WEAVESIM_H
#define WEAVESIM_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------------------------------ status codes */
#define WS_OK 0
#define WS_ERR_ARG -1        /* malformed argument or model (GpuSolver throws Error: web/js/solver_gpu.js:70) */
#define WS_ERR_CUDA -2       /* a CUDA call failed */
#define WS_ERR_NOMEM -3      /* device memory budget exhausted (admission refused) */
#define WS_ERR_STATE -4      /* call not valid in the current state (e.g. changed clamps: solver_gpu.js:325) */
#define WS_ERR_NODEV -5      /* no CUDA device: the library has no CPU fallback */

/* per-instance status in ws_control.status */
#define WS_RUNNING 0
#define WS_CONVERGED 1
#define WS_MAX_ITER 2
#define WS_NONFINITE 3
#define WS_DONE 4        /* the load protocol (ws_protocol) recorded its last increment */

/* precision of a solver context (one template instantiation of every kernel) */
#define WS_PREC_F64 0        /* FP64 everywhere */
#define WS_PREC_MIXED 1      /* FP32 element math, two-float positions/frames, FP64 strain / relative rotation /
                                contact gap, slide coordinates and reductions */
#define WS_PREC_F32 2        /* naive FP32 everywhere */

/* execution form */
#define WS_FORM_CTA 0        /* persistent fused kernel, one thread block per instance (batched) */
#define WS_FORM_GRID 1       /* persistent fused kernel, one instance over a cooperative grid with bounded grid barriers */
#define WS_FORM_PLAIN 2      /* one kernel per phase per iteration, one instance (the plain GPU form) */

/* ------------------------------------------------------------------------------------------------ parameters */
/* Solver and contact parameters that the DR step reads.  Defaults: params.js:8-23 (SOLVER, CONTACT).
 * Units are the model's (these bindings use SI: m, N, Pa). */
typedef struct ws_params {
  double mass_scale;      /* SOLVER.mass_scale 1.5 */
  double damping;         /* SOLVER.damping 1.0 */
  double tol;             /* SOLVER.tol 1e-4 (relative residual, solver_cpu.js:829-837) */
  int32_t kinetic_damping;/* SOLVER.kinetic_damping 1 */
  int32_t warmup_iter;    /* SOLVER.warmup_iter 300 */
  int32_t max_iter;       /* SOLVER.max_iter 5000 */
  int32_t contacts;       /* CpuSolver {contacts}: 1 = crossings active (solver_cpu.js:662,685) */
  double strength;        /* CONTACT.strength: normal penalty [force/length] */
  double stick_strength;  /* CONTACT.stick_strength: stick spring [force/length] */
  double torsion_factor;  /* CONTACT.torsion_factor 1.0 */
  double epsilon;         /* CONTACT.epsilon: slide step limit per iteration [length] */
  int32_t ramp_iter;      /* CONTACT.ramp_iter 1500 */
  int32_t disp_ramp_iter; /* prescribed support motion: anchored translations reach ws_model.anchor_target after this
                             many iterations, linearly (0: at the first iteration).  An extension: the reference's
                             anchors hold the position they have (solver_cpu.js:764,781). */
  double slip_rate;       /* CONTACT.slip_rate 1.0 */
  double edge_threshold;  /* CONTACT.edge_threshold 0.5: a side bears on an edge when |tanh(n·X/0.03) tanh(n·Y/0.03)| exceeds
                             it (W1 classification, solver_cpu.js:231-271) */
  /* contact extensions (params.js:10-14); all off by default */
  int32_t augmented;      /* CONTACT.augmented 0: augmented-Lagrangian gap, Fn = max(0, λ + k_n·pen) (solver_cpu.js:414-418) */
  int32_t al_every;       /* CONTACT.al_every 600: Uzawa update of λ every al_every iterations after the ramp
                             (solver_cpu.js:819-821, 484-506) */
  int32_t rot_friction;   /* CONTACT.rot_friction 0: W2 rotational friction about the contact normal (solver_cpu.js:347-379) */
  int32_t seat_law;       /* CONTACT.seat_law: 0 'off', 1 'L1' (W3 directional seat law, solver_cpu.js:283-344) */
  int32_t seat_gap;       /* CONTACT.seat_gap 1: the seat depth closes the section gap (solver_cpu.js:410) */
  int32_t dent_after_iter;/* CONTACT.dent_after_iter -1: seats form from this iteration on; -1 = warmup_iter + ramp_iter of
                             the model the instance was created from (solver_cpu.js:329,686) */
  double rot_factor;      /* CONTACT.rot_factor 1.0: W2 moment limit rot_factor·μ·|Fn|·r_eq */
  double dent_rate;       /* CONTACT.dent_rate 0.01: share of the estimated seat depth added per iteration */
  /* the ground (scene.floor, Floor in solver_cpu.js:509-634): a plane at height floor_z that the sections cannot pass,
   * penalty k_n = strength, stick spring k_t = stick_strength (with the contact ramp), Coulomb coefficient floor_mu */
  int32_t floor;          /* 0 none, 1 on; a model with a ground must also have an anchor (the rigid-body freedoms of a
                             model that only the ground holds are not built) */
  int32_t pad1;
  double floor_z;         /* height of the plane */
  double floor_mu;        /* friction coefficient on the ground */
} ws_params;

/* UTM replay protocol of one instance: the GpuSolver protocol (web/js/wgsl.js:1048-1093, set up by
 * solver_gpu.js:256-318 and driven by calibrate.js:438-515).  Per load increment: settle (at most `settle`
 * iterations, fewer once the residual meets the tolerance), then average the probe's travel along `axis` and the
 * reaction along `axis` over `avg` iterations, record them, and apply the next value of the schedule: a force on the
 * probe (mode 1) or the probe's position P0 + value·axis, the probe held there (mode 2; P0 = the probe's position when
 * the instance was created or uploaded).  Convergence does not stop such an instance; it stops with WS_DONE after the
 * last increment (or at max_iter, which must therefore cover n_inc × (settle + avg)). */
#define WS_PROTOCOL_MAX_INC 64
typedef struct ws_protocol {
  int32_t mode;           /* 0 none, 1 force control, 2 displacement control */
  int32_t probe;          /* probe node */
  int32_t n_inc;          /* increments (1..WS_PROTOCOL_MAX_INC) */
  int32_t settle;         /* settling iterations per increment */
  int32_t avg;            /* iterations the read-out is averaged over */
  int32_t pad0;
  double axis[3];         /* probe axis (unit vector) */
  double sched[WS_PROTOCOL_MAX_INC];   /* force [N] (mode 1) or travel [m] (mode 2) of each increment */
} ws_protocol;

/* The model of one instance: the flat state of buildState (web/js/model.js:10-75), the section stiffness per segment
 * (strandStiffness, model.js:236-252), the loads (Loads, model.js:191-231), the resolved anchors (anchorMasks /
 * Anchors, model.js:150-189) and the crossings (PolylineContact constructor, solver_cpu.js:62-96), before the goals
 * (masses, inertias, clamp joints) and the contact initialisation, which every consumer builds itself. */
typedef struct ws_model {
  int32_t n, m, p, n_strands, K;
  int32_t pad0;
  const double *X;            /* [3n] current positions */
  const double *X0;           /* [3n] displacement origin */
  const double *Q;            /* [4m] segment frames (w, x, y, z); columns of R = [X width | Y normal | Z tangent] */
  const double *l0;           /* [m] rest lengths */
  const int32_t *seg_i0;      /* [m] first node of segment */
  const int32_t *seg_i1;      /* [m] second node of segment */
  const int32_t *seg_offset;  /* [n_strands+1] first segment of every strand */
  const int32_t *joint_seg0;  /* [p] segment a of joint */
  const int32_t *joint_seg1;  /* [p] segment b of joint */
  const double *joint_len;    /* [p] Voronoi length l̄ */
  const double *omega0;       /* [3p] rest curvature Ω0 (NULL: zeros) */
  const double *EA, *EIx, *EIy, *GJ, *GA;   /* [m] section stiffness */
  const double *load_const;   /* [3n] constant loads (self-weight, UDL, world point loads) */
  int32_t n_local_loads;
  int32_t n_anchors;
  const int32_t *local_load_node;  /* [n_local_loads] */
  const double *local_load_F;      /* [3 n_local_loads] in the node frame */
  const int32_t *anchor_node;      /* [n_anchors] in resolution order */
  const uint8_t *anchor_mask;      /* [n_anchors] bit k fixes DOF k of [X Y Z rX rY rZ] */
  const double *anchor_target;     /* [3 n_anchors] target positions of the anchored nodes (NULL: they stay) */
  const int32_t *cross_strand;     /* [2K] strand of side A, side B of every crossing (knots in sorted edge order) */
  const double *cross_wk, *cross_hk;   /* [2K] section width / height of each side */
  const double *cross_u;           /* [2K] slide coordinates (global u along the strand) */
  const double *cross_nprev;       /* [3K] persistent contact normal */
  const uint8_t *cross_enabled;    /* [K] */
  const uint8_t *cross_locked;     /* [K] */
  const double *cross_mu;          /* [K] Coulomb coefficient per crossing (the reference has one contact.mu) */
  const double *cross_fc90, *cross_E90, *cross_H;  /* [2K] timber of each side across the grain: crushing strength,
                                        modulus, hardness (PolylineContact's matOf, solver_cpu.js:71-76); NULL: the
                                        reference's defaults 8, 800, 30 (N/mm²) */
  ws_params params;
  const ws_protocol *protocol;     /* NULL: relax to convergence */
  const double *node_w, *node_h;   /* [n] section width / height at every node (its lath group), for the ground's
                                      clearance; needed when params.floor is on */
} ws_model;

/* per-instance control block, written by the device after every iteration (the CT struct of the WebGPU solver,
 * web/js/wgsl.js:154-172, read by GpuSolver.readControl, solver_gpu.js:374-386) */
typedef struct ws_control {
  int32_t iter;        /* DR iterations done */
  int32_t status;      /* WS_RUNNING / WS_CONVERGED / WS_MAX_ITER / WS_NONFINITE / WS_DONE */
  int32_t rollbacks;   /* kinetic-damping resets since creation */
  int32_t pending_zero;/* 1: the last iteration rolled back (velocities are zero, state is the previous one) */
  double ke;           /* kinetic energy of the last iteration (0 after a reset) */
  double ke_prev;      /* kinetic-energy peak tracker (CpuSolver.kePrev) */
  double residual;     /* max(force part, torque part); +inf during the warm-up */
  double res_force, res_torque, fref;
  double e_stretch, e_shear, e_bend, e_twist, e_contact;
  int32_t utm_inc;     /* load increments recorded (ws_protocol) */
  int32_t utm_phase;   /* 0 settling, 1 averaging, 2 finished */
  double e_floor;      /* the ground's spring energy (Floor.energy) */
  double t_start_ms;   /* batched form: when the instance's block (or cluster) took it up in the last ws_step, and */
  double t_end_ms;     /* when it left it, in ms after the earliest start of that step (device timer); other forms 0 */
} ws_control;

/* ------------------------------------------------------------------------------------------------ errors */
/* copies the message of the last failing call on this thread into buf (always NUL-terminated); returns its length */
int ws_last_error(char *buf, size_t n);
/* number of visible CUDA devices (0 when there is none) */
int ws_device_count(void);

/* ------------------------------------------------------------------------------------------------ scenes */
/* Synthetic Kagome gridshell on a hexagonal plan: a triangular lattice clipped to a hexagon of `side` triangle edges
 * (the tri_lattice pattern of examples/make_meshes.py:13-29), traced into laths by buildTopology
 * (web/js/topology.js:78-87), subdivided, pre-offset and framed (topology.js:214-345), and flattened by buildState
 * (model.js:10-75).  Laths per family = 2·side; triangle edge a = family spacing·2/√3. */
typedef struct ws_kagome_cfg {
  int32_t side;              /* hexagon side in triangle edges (laths per family / 2) */
  int32_t subdivisions;      /* WEAVE.subdivisions: segments between neighbouring knots */
  double edge;               /* triangle edge a [m] */
  double width, height;      /* lath section [m] */
  double E, G, density;      /* material [Pa, Pa, kg/m^3] */
  double mu;                 /* Coulomb coefficient (all crossings) */
  double mu_lo, mu_hi;       /* if mu_hi > mu_lo: per-crossing mu ~ U(mu_lo, mu_hi) from the seed */
  double inward;             /* radial inward displacement of the perimeter lath ends [m] (scales the plan) */
  double lift;               /* support ends lifted 0..lift [m] by a smooth seeded field (0: none) */
  double z_noise;            /* std. dev. of the seeded z-noise of every node [m] */
  int32_t gravity;           /* 1: self-weight on */
  uint32_t seed;             /* xoshiro128** seed (web/js/rng.js:9-27) */
  ws_params params;
} ws_kagome_cfg;

typedef struct ws_scene ws_scene;   /* owns the arrays of one ws_model */

/* A scene from a triangle mesh: the scene.json path of the reference (Scene.fromJSON, web/js/scene.js:142-190;
 * Mesh.fromBytes, mesh.js:23-31; buildTopology, topology.js; Anchors / Loads / strandStiffness, model.js:112-252), with
 * the file reading, the vertex weld and the unit conversions done by the caller (weave-sim_b200/scenefile.py). */
enum { WS_SEL_FRAME = 0, WS_SEL_ALL_START = 1, WS_SEL_ALL_END = 2, WS_SEL_ALL_ENDS = 3, WS_SEL_STRAND = 4, WS_SEL_BOUNDARY = 5 };
/* one lath group: its section, stiffness, prestress shares, self-weight per length and material across the grain,
 * in the same meaning as the ws_mesh_cfg fields of those names */
typedef struct ws_lath_group {
  double width, height;
  double EA, EIx, EIy, GJ, GA;
  double activation[3];
  double line_weight;
  double fc90, E90, H;
} ws_lath_group;
typedef struct ws_mesh_cfg {
  int32_t n_vertices, n_faces;
  const double *vertices;      /* [3 n_vertices] welded and scaled (Mesh.fromBytes) */
  const int32_t *faces;        /* [3 n_faces] consistently oriented triangles */
  int32_t subdivisions;        /* weave.subdivisions */
  int32_t half_height;         /* weave.offset_mode == 'half_height' */
  int32_t seed_strand_phase;   /* weave.seed_strand_phase */
  int32_t n_flips;
  const int32_t *flips;        /* [2 n_flips] weave.flip_knots (strand, knot) */
  double overhang;             /* weave.overhang; without it the boundary crossings carry no contact */
  double width, height;        /* section */
  double EA, EIx, EIy, GJ, GA; /* section stiffness times the beam factors (sectionStiffness × beamFactors) */
  double activation[3];        /* prestress shares (flat, edge, twist): rest curvature (1 − a) × the as-built one */
  double line_weight;          /* self-weight per length in scene units (UnitSystem.selfWeightLineLoad); 0: none */
  double gravity_dir[3];
  int32_t udl_on;              /* 1: loads.udl per length, on the nodes' tributary lengths; 2: per area, the mesh's
                                  area shared in proportion to the tributary lengths (Loads, model.js:213-220) */
  int32_t pad0;
  double udl[3];
  double mu;                   /* contact.mu */
  double fc90, E90, H;         /* material across the grain */
  int32_t n_anchors, pad1;
  const int32_t *anchor_kind;  /* WS_SEL_* per selector, in the scene's order */
  const int32_t *anchor_id;    /* [2 n_anchors] (strand, knot) of a frame, the strand of WS_SEL_STRAND */
  const uint8_t *anchor_mask;  /* [n_anchors] bit k fixes DOF k of [X Y Z rX rY rZ] */
  int32_t n_loads, pad2;
  const int32_t *load_frames;  /* [2 n_loads] */
  const double *load_F;        /* [3 n_loads] */
  const uint8_t *load_local;   /* [n_loads] 1: in the node frame */
  ws_params params;
  /* lath groups of a hybrid weave (scene.hybrid, web/js/scene.js:50-68; strandStiffness, model.js:236-252): group g
   * >= 2 of strand s (assign_strand[i] = s, assign_group[i] = g) takes groups[g - 2]'s section, stiffness,
   * activation, self-weight and material across the grain for its segments, joints (the group of the joint's first
   * segment), crossing sides and nodes, and its height for the knot offsets (the mean of the two strands' heights,
   * topology.js:225); every other strand takes the fields above.  n_groups = 0: one group. */
  int32_t n_groups, n_assign;
  const struct ws_lath_group *groups;
  const int32_t *assign_strand, *assign_group;
} ws_mesh_cfg;
int ws_scene_mesh(const ws_mesh_cfg *cfg, ws_scene **out);


/* defaults: params.js:8-23 converted to SI (strength 1e4 N/mm = 1e7 N/m, epsilon 15 mm) */
void ws_params_default(ws_params *out);
int ws_scene_kagome(const ws_kagome_cfg *cfg, ws_scene **out);
/* Stand-alone laths with optional knots (topologyFromPolylines, topology.js:348-363; the test fixtures of
 * web/tests/cases.mjs:10-28).  Strand s has node_count[s] points in `points`, optional per-node normals hints,
 * knot_count[s] knot rows in `knot_rows`; knots pair frame (sa, ka) with (sb, kb).  Anchors by frame (s, k) and
 * DOF mask; point loads by frame with a world (local = 0) or node-frame (local = 1) force. */
typedef struct ws_polyline_cfg {
  int32_t n_strands;
  const int32_t *node_count;      /* [n_strands] */
  const double *points;           /* [3 Σ node_count] */
  const double *normals;          /* [3 Σ node_count] or NULL (hint (0, 0, 1)) */
  const int32_t *knot_count;      /* [n_strands] or NULL (rows 0 and n-1) */
  const int32_t *knot_rows;       /* [Σ knot_count] */
  int32_t n_knots;
  const int32_t *knots;           /* [4 n_knots] sa, ka, sb, kb */
  double thickness;               /* pre-offset thickness (unused for stand-alone laths) */
  int32_t n_anchors;
  const int32_t *anchor_frames;   /* [2 n_anchors] */
  const uint8_t *anchor_masks;    /* [n_anchors] */
  int32_t n_loads;
  const int32_t *load_frames;     /* [2 n_loads] */
  const double *load_F;           /* [3 n_loads] */
  const uint8_t *load_local;      /* [n_loads] */
  double width, height, E, G, density;
  double mu;
  int32_t gravity;
  ws_params params;
} ws_polyline_cfg;
int ws_scene_polylines(const ws_polyline_cfg *cfg, ws_scene **out);
/* the model view of a scene (pointers stay valid until ws_scene_free) */
const ws_model *ws_scene_model(const ws_scene *s);
/* per-strand node offsets [n_strands+1] and the span of the plan (largest extent of X0 in x or y) */
const int32_t *ws_scene_node_offset(const ws_scene *s);
double ws_scene_span(const ws_scene *s);
void ws_scene_free(ws_scene *s);

/* The goals the device will use for a model, built on the host (no GPU needed): node masses [n], static frame stiffness
 * per body axis [3m], slide coordinates and contact normals after the contact initialisation [2K], [3K], the torque
 * residual's reference length (CpuSolver._buildGoals, solver_cpu.js:670-710; PolylineContact.initialize,
 * solver_cpu.js:99-139).  Any output pointer may be NULL. */
int ws_model_goals(const ws_model *model, double *mass, double *k_rot_static, double *u, double *nprev, double *l_ref);

/* ------------------------------------------------------------------------------------------------ solver */
typedef struct ws_ctx ws_ctx;

typedef struct ws_opts {
  int32_t precision;    /* WS_PREC_* */
  int32_t form;         /* WS_FORM_* */
  int32_t threads;      /* threads per block of the batched form (0: 512 with shared-memory state, 256 with global) */
  int32_t device;       /* CUDA device ordinal */
  uint64_t budget_bytes;/* device memory this context may take (0: no limit) */
  int32_t cta_state;    /* batched form: WS_CTA_AUTO keeps each instance's changing state in shared memory when every
                           instance of the batch fits a thread block's shared memory, else in global memory;
                           WS_CTA_GLOBAL always in global memory */
  int32_t side_order;   /* WS_SIDES_AUTO: the short-slide side order when the slide limit (contact epsilon) is under half
                           the shortest segment of the strands with crossings, else the general order;
                           WS_SIDES_GENERAL: always the general order */
  int32_t wide_cluster; /* batched form: thread blocks (of 512 threads) in the cluster that relaxes one wide instance,
                           2..8; 1: every instance in one block; 0: the default (2) */
  int32_t wide_min;     /* batched form: an instance is wide when its nodes + segments reach this (0: the default,
                           32768); an instance with a load protocol is never wide */
  int32_t tune;         /* 1: the launch shape (the fields above from threads on, and the plain form's launch mode) is
                           the autotuner's: taken from its cache for the batch's size bucket on this device, or found
                           by timing every candidate shape on this batch at creation (the state is restored after the
                           trials); 0: the fields above as given */
} ws_opts;

/* A launch shape.  The batched form: threads per block of the one-block kernels (128, 256, 512), cta_state
 * (WS_CTA_AUTO or WS_CTA_GLOBAL), wide_cluster (1: no wide instances, else blocks of 512 threads per wide instance's
 * cluster) and wide_min (nodes + segments from which an instance is wide).  The plain form: plain_launch (0 forked
 * graph branches, 1 one launch a phase with block roles, 2 one kernel a phase).  source: 0 as given by the options, 1
 * found by the tuner when the context was made, 2 from the tuner's cache.  trial_ms: the time of the shape's trial run
 * (tuned shapes), default_ms: that of the default shape in the same trials, trials: candidates timed. */
typedef struct ws_shape {
  int32_t threads, cta_state, wide_cluster, wide_min, plain_launch, source, trials, pad0;
  double trial_ms, default_ms;
} ws_shape;
enum { WS_SIDES_AUTO = 0, WS_SIDES_GENERAL = 1 };
enum { WS_CTA_AUTO = 0, WS_CTA_GLOBAL = 1 };

/* Builds the goals of every instance on the host (masses, inertias, clamps: CpuSolver._buildGoals,
 * solver_cpu.js:670-710; contact initialisation: PolylineContact.initialize, solver_cpu.js:99-139) and uploads the
 * batch.  Replaces `new GpuSolver(device, models, opts)` (solver_gpu.js:65-130); unlike it, the instances need not
 * share one topology. */
int ws_create(const ws_model *const *models, int32_t n_instances, const ws_opts *opts, ws_ctx **out);
/* Runs up to n_iter DR iterations (CpuSolver.step, solver_cpu.js:737-841) on every instance whose mask byte is non-zero
 * (NULL: all), each stopping at its own convergence; the control blocks of all instances go to ctl[n_instances]
 * (NULL: not read).  Replaces GpuSolver.step (solver_gpu.js:338-361).  Asynchronous on the context's stream unless
 * ctl is given. */
int ws_step(ws_ctx *ctx, int32_t n_iter, const uint8_t *instance_mask, ws_control *ctl);
int ws_read_control(ws_ctx *ctx, ws_control *ctl);
/* State of one instance, host buffers sized by its model (any pointer may be NULL).  Replaces GpuSolver.download
 * (solver_gpu.js:431-503). */
typedef struct ws_state_out {
  double *X;       /* [3n] */
  double *Q;       /* [4m] */
  double *V;       /* [3n] */
  double *W;       /* [3m] body angular velocities */
  double *u;       /* [2K] */
  double *nprev;   /* [3K] */
  double *slip;    /* [K] accumulated slip */
  uint8_t *stuck;  /* [K] */
  uint8_t *state;  /* [K] 1 = slipping in the last iteration */
  double *Fn;      /* [K] */
  double *Ft;      /* [K] */
  double *gap;     /* [K] */
  double *N;       /* [m] axial force */
  double *Vsh;     /* [2m] shear forces */
  double *M;       /* [3p] joint moments */
  double *reactions; /* [3n] */
  /* W1 classification of the last evaluation (PolylineContact._classify, solver_cpu.js:231-271; buildResults,
   * solver_cpu.js:903-905) */
  uint8_t *ctype;  /* [K] 0 face-face, 1 edge-face, 2 edge-edge */
  double *theta;   /* [K] crossing angle asin|t_A × t_B| */
  double *phi;     /* [2K] roll of each side's section against the contact plane */
  double *area;    /* [K] nominal contact area */
  double *pressure;/* [K] */
  double *util;    /* [K] pressure against hardness (face-face), fc90 (edge-face) or 1 (edge-edge) */
  /* contact extensions (buildResults, solver_cpu.js:906-908) */
  double *lambda;  /* [K] augmented-Lagrangian multiplier λ */
  double *dent;    /* [K] seat depth: the dents of both sides + the edge-on-face embedment */
  double *M_rot;   /* [K] W2 scissor moment about the contact normal */
  double *rot_slip;/* [K] accumulated W2 rotational slip [rad] */
  /* load protocol read-out (GpuSolver.readOutputs, solver_gpu.js:407-416): per recorded increment the mean probe
   * travel along the axis, the mean reaction along the axis, the applied value and the iteration */
  double *utm;     /* [4 WS_PROTOCOL_MAX_INC] */
  /* the ground (Floor.F / Floor.state, solver_cpu.js:541-546) */
  double *floor_F; /* [3n] the ground's force on every node */
  uint8_t *floor_state; /* [n] 0 clear of the ground, 1 stuck, 2 sliding */
  /* results post-processing on the device (buildResults, solver_cpu.js:878-898; fields.js nodeValues) */
  double *seg_M;   /* [3m] Mx, My, T of every segment, from the moments of its end joints and clamps */
  double *node_M;  /* [4n] Mx, My, T, N at the nodes: the mean of a node's segments along its strand */
  double *disp;    /* [3n] X − X0 (X0: the displacement origin, moved by ws_internalize) */
} ws_state_out;
int ws_download(ws_ctx *ctx, int32_t instance, ws_state_out *out);
/* Uploads positions and frames (and zeroes velocities) of one instance from host buffers: a warm start from a state the
 * caller holds (GpuSolver.upload, solver_gpu.js:189-198).  X [3n], Q [4m]; u [2K] may be NULL (kept). */
int ws_upload_state(ws_ctx *ctx, int32_t instance, const double *X, const double *Q, const double *u);
/* Warm start with new parameters (rebuildGoals + GpuSolver.updateParams, solver_cpu.js:719-732,
 * solver_gpu.js:323-333): stiffness, loads, contact parameters and per-crossing mu of `model` replace the
 * instance's; positions, frames, contact state stay on the device; masses and inertias are rebuilt from the current
 * state; the kinetic-energy peak and the convergence flag are reset.  Anchored nodes move to model->X where their
 * translation is fixed (prescribed displacement).  The topology must be the instance's. */
int ws_set_params(ws_ctx *ctx, int32_t instance, const ws_model *model);
/* Replaces instance b by a new model with the same element counts (a serving slot taking its next request): goals,
 * contact initialisation, state and control are rebuilt from `model` and the iteration count restarts at 0.  The
 * other instances keep running; no device memory is allocated. */
int ws_load_instance(ws_ctx *ctx, int32_t instance, const ws_model *model);
/* current geometry becomes the displacement origin; slip counters restart (CpuSolver.internalize, solver_cpu.js:868;
 * GpuSolver.internalize, solver_gpu.js:507-520) */
int ws_internalize(ws_ctx *ctx, int32_t instance);
/* Allocation-free relaxation of one small instance, for callers that cannot allocate device memory themselves (a
 * framework that owns the GPU's memory through its own pool, a serving process that must not allocate once running).
 * No counterpart in the reference.  The instance's whole device footprint lives in one static array of
 * WS_NOALLOC_SCRATCH_BYTES that every GPU loading this library holds until exit; models that need more are rejected
 * with WS_ERR_ARG.  The call builds the goals, clears the array, uploads `model`, runs n_iter iterations of the batched
 * kernel on `stream` (NULL: the default stream; a stream of another device than the current one is rejected with
 * WS_ERR_ARG), waits for them and fills `out` and `ctl` (either may be NULL).  The result is bit for bit that of
 * ws_create with opts.form = WS_FORM_CTA, opts.cta_state = 1 (global state) and the same `threads` (0 here: 256),
 * followed by ws_step and ws_download.  The call allocates no device memory; the array itself is reserved when the
 * driver loads the library's device code on a device, which with CUDA's lazy module loading happens at the first call
 * there: make one call (n_iter = 0 will do) at start-up, before a pool takes the device's memory, and before any stream
 * capture.  Every call looks up the array's device address on the current device (cudaGetSymbolAddress), so a device
 * reset in between is harmless.  Every call shares the array and leaves its contents behind: calls from this process
 * take turns on a lock, but calls whose GPU work overlaps (several processes, or this entry point mixed with raw
 * launches that touch the array) race. */
#define WS_NOALLOC_SCRATCH_BYTES (16u << 20)
int ws_relax_noalloc(const ws_model *model, int32_t precision, int32_t n_iter, int32_t threads, void *stream,
                     ws_state_out *out, ws_control *ctl);
/* CUDA stream of the context (cudaStream_t) */
void *ws_stream(ws_ctx *ctx);
/* side order in use: 1 the short-slide order (the crossing sides are ranked inside the element kernel and a side moves
 * at most one segment per iteration), 0 the general order (a separate ranking kernel).  No counterpart in the
 * reference, whose GPU form re-sorts nothing (it accumulates with atomics). */
int ws_side_order(const ws_ctx *ctx);
/* 1 when the batched form holds its instances in shared memory (the resident form), else 0.  No counterpart in the
 * reference. */
int ws_cta_resident(const ws_ctx *ctx);
/* batched form: the number of wide instances (each relaxed by a thread-block cluster) and, in *cluster (may be NULL),
 * the blocks per cluster (0 when there are none) */
int ws_wide_instances(const ws_ctx *ctx, int32_t *cluster);
/* the launch shape the context runs (ws_shape) */
int ws_get_shape(const ws_ctx *ctx, ws_shape *out);
/* The autotuner's cache, keyed by a batch's size bucket on a device (ws_tune_key: form, precision, variants,
 * instance count, largest instance and total work in half-octave steps; no device needed).  ws_tune_candidates lists
 * the shapes the tuner times for such a batch: stage 1 (block size and state placement, no wide instances) when
 * `after` is NULL, else stage 2 (cluster shapes and thresholds at the stage-1 winner `after`); it returns how many there
 * are and writes up to `cap` of them.  ws_tune_cache_get returns 1 and the shape when the key is cached, else 0; _put
 * stores one (also appended to the file WEAVESIM_TUNE_CACHE names, when set); _clear empties the process's cache. */
int ws_tune_key(const ws_model *const *models, int32_t n_instances, const ws_opts *opts, const char *device, char *buf,
                size_t cap);
int ws_tune_candidates(const ws_model *const *models, int32_t n_instances, const ws_opts *opts, const ws_shape *after,
                       ws_shape *out, int32_t cap);
int ws_tune_cache_get(const char *key, ws_shape *out);
int ws_tune_cache_put(const char *key, const ws_shape *shape);
int ws_tune_cache_clear(void);
/* device bytes held by the context */
uint64_t ws_device_bytes(const ws_ctx *ctx);
/* GPU time of the last ws_step (ms, CUDA events on the context's stream) and the number of kernel launches it made */
int ws_last_step_stats(const ws_ctx *ctx, double *ms, int64_t *launches);
int ws_destroy(ws_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
