/* natsel_gpu.h -- C ABI of the B200 rigid-body step (libnatsel_gpu.so).
 *
 * The library is a drop-in for the reference engine's per-step rigid-body solve
 * (reference: src/simulation/solver_integration.rs:807 World::step and the
 * stages it calls: collide_pass.rs:164 collide, constraint_graph.rs:113
 * add_contact_to_graph, solver_prepare.rs:269 prepare_all_contacts,
 * solver_stages.rs:543 solve_constraint_stages, solver_integration.rs:435
 * finalize_bodies, plus the broadphase pair update contact_creation.rs:901).
 * Scene construction mirrors the reference World API so a host engine builds
 * the same bodies/shapes/joints in the same order and gets the same ids.
 *
 * Plain C types only. Every call returns an int status (NS_OK == 0) unless
 * documented otherwise; ns_last_error() gives a message. Calls on one world
 * must be serialised by the caller (the reference World is Send, not Sync);
 * distinct worlds may be used from distinct threads.
 */
#ifndef NATSEL_GPU_H
#define NATSEL_GPU_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum {
  NS_OK = 0,
  NS_ERR_INVALID = 1,     /* bad argument or call order */
  NS_ERR_CUDA = 2,        /* CUDA runtime error (message in ns_last_error) */
  NS_ERR_CAPACITY = 3,    /* a device capacity (contacts, pairs) was exceeded */
  NS_ERR_TIMEOUT = 4,     /* a bounded grid barrier gave up; the step result is invalid */
  NS_ERR_NONFINITE = 5,   /* finalize found a NaN/Inf velocity, position or rotation (reported by
                             the next synchronising call; the world stays in error) */
  NS_ERR_UNSUPPORTED = 6  /* feature outside the implemented path (e.g. sleeping) */
};

enum { NS_STATIC_BODY = 0, NS_KINEMATIC_BODY = 1, NS_DYNAMIC_BODY = 2 };

typedef struct ns_world ns_world;

/* World settings. Defaults follow the reference World::new (world_runtime.rs:1243-1272). */
typedef struct {
  float gravity[3];            /* (0,-10,0) */
  int enable_sleep;            /* must be 0: sleeping islands are outside this path */
  int enable_continuous;       /* 1: fast dynamic bodies are swept against static shapes after
                                  finalize and moved back to the time of impact (continuous.rs:337);
                                  fast bullets then against dynamic bodies too */
  int enable_warm_starting;    /* 1 */
  float contact_hertz;         /* 30 */
  float contact_damping_ratio; /* 10 */
  float contact_speed;         /* 3 m/s */
  float max_linear_speed;      /* 400 m/s */
  float restitution_threshold; /* 1 m/s */
  int restitution_iterations;  /* 2 */
  float joint_hertz;           /* 60 (JointDef default, joint_defs.rs:44) */
  float joint_damping_ratio;   /* 2 */
  int contact_capacity;        /* 0 = automatic (8 per shape + 4096) */
  int solver_blocks;           /* solver launch: 0 = automatic (a grid over every SM for sub-worlds
                                  or a world of 2048 awake bodies or more, else one 16-CTA cluster
                                  on B200); 1..16 = one thread-block cluster of that many CTAs;
                                  > 16 = cooperative grid of that many blocks (capped at what fits
                                  co-resident) */
  int device;                  /* CUDA device ordinal */
} ns_world_def;

/* Body definition (types/body_def.rs BodyDef). */
typedef struct {
  int type;                    /* NS_STATIC_BODY, NS_KINEMATIC_BODY (moves at its own velocity,
                                  zero mass, collides with dynamic bodies only) or NS_DYNAMIC_BODY */
  double position[3];
  float rotation[4];           /* x, y, z, s */
  float linear_velocity[3];
  float angular_velocity[3];
  float linear_damping, angular_damping, gravity_scale;
  int enable_sleep;            /* stored as a body flag; sleeping itself is not simulated */
  int is_bullet;               /* body_def.rs:74: when fast, swept against dynamic bodies too */
} ns_body_def;

/* Shape definition (types/shape_def.rs ShapeDef with one surface material). */
typedef struct {
  float density, friction, restitution, rolling_resistance;
  uint64_t category_bits, mask_bits;
  int group_index;
} ns_shape_def;

void ns_default_world_def(ns_world_def* def);
/* Creates a world; returns NULL on failure (message via ns_last_error(NULL)). */
ns_world* ns_world_create(const ns_world_def* def);
void ns_world_destroy(ns_world* world);
const char* ns_last_error(const ns_world* world);

/* Scene construction (replaces World::create_body world_runtime.rs:1506,
 * create_hull_shape(make_box_hull) shape_creation.rs:559 / hull.rs:853,
 * create_sphere_shape :504, create_capsule_shape :522,
 * create_revolute_joint revolute_joint.rs:162). Returns the new id (>= 0) or -1. */
int ns_create_body(ns_world* world, const ns_body_def* def);
int ns_create_box_shape(ns_world* world, int body, const ns_shape_def* def, float hx, float hy, float hz);
int ns_create_sphere_shape(ns_world* world, int body, const ns_shape_def* def, const float center[3],
                           float radius);
int ns_create_capsule_shape(ns_world* world, int body, const ns_shape_def* def, const float center1[3],
                            const float center2[3], float radius);
/* frame = position xyz + rotation xyzs, local to each body's origin. The joint's softness is the
 * world's joint_hertz / joint_damping_ratio; max_motor_torque > 0 enables a motor of speed 0
 * (a drag torque). ns_create_revolute_joint_def takes every field instead. */
int ns_create_revolute_joint(ns_world* world, int body_a, int body_b, const float frame_a[7],
                             const float frame_b[7], int enable_limit, float lower_angle,
                             float upper_angle, int enable_spring, float hertz, float damping_ratio,
                             float max_motor_torque, int collide_connected);

/* RevoluteJointDef (types/joint_defs.rs:154, with its JointDef base :30; the base's force and
 * torque thresholds and draw scale belong to joint events and debug draw, outside this path).
 * The rotation axis is the z axis of the local frames. */
typedef struct {
  int body_a, body_b;
  float local_frame_a[7], local_frame_b[7]; /* position xyz + rotation xyzs */
  float constraint_hertz;                    /* 60 */
  float constraint_damping_ratio;            /* 2 */
  int collide_connected;                     /* 0 */
  float target_angle;                        /* spring rest angle, radians */
  int enable_spring;
  float hertz, damping_ratio;
  int enable_limit;
  float lower_angle, upper_angle;
  int enable_motor;
  float max_motor_torque, motor_speed;
} ns_revolute_joint_def;
/* Defaults of RevoluteJointDef::default (everything off, identity frames, bodies -1). */
void ns_default_revolute_joint_def(ns_revolute_joint_def* def);
/* create_revolute_joint (revolute_joint.rs:161) with the whole definition. Returns the joint id
 * (>= 0) or -1. */
int ns_create_revolute_joint_def(ns_world* world, const ns_revolute_joint_def* def);

/* SphericalJointDef (types/joint_defs.rs:169, with its JointDef base :30): a ball-and-socket joint
 * at the frames' origins; the cone limit bounds the angle between the frames' z axes, the twist
 * limit the rotation about body B's z axis, the spring pulls the relative rotation to
 * target_rotation and the motor drives the relative angular velocity to motor_velocity. */
typedef struct {
  int body_a, body_b;
  float local_frame_a[7], local_frame_b[7]; /* position xyz + rotation xyzs */
  float constraint_hertz;                    /* 60 */
  float constraint_damping_ratio;            /* 2 */
  int collide_connected;                     /* 0 */
  int enable_spring;
  float hertz, damping_ratio;
  float target_rotation[4];                  /* xyzs, identity */
  int enable_cone_limit;
  float cone_angle;
  int enable_twist_limit;
  float lower_twist_angle, upper_twist_angle;
  int enable_motor;
  float max_motor_torque;
  float motor_velocity[3];
} ns_spherical_joint_def;
void ns_default_spherical_joint_def(ns_spherical_joint_def* def);
/* spherical_joint.rs:119 create_spherical_joint. Returns the joint id (>= 0) or -1. */
int ns_create_spherical_joint_def(ns_world* world, const ns_spherical_joint_def* def);

/* Batched worlds (no counterpart in the reference, which steps one world at a time): a world
 * can hold several independent sub-worlds that are stepped together by every ns_world_step.
 * Sub-world 0 exists from creation; ns_world_begin_subworld starts the next one and returns
 * its index (-1 after the first step). Bodies created afterwards belong to it, and shapes and
 * joints can only be added to bodies of the newest sub-world, so each sub-world's bodies,
 * shapes and joints have contiguous ids. Bodies of different sub-worlds never collide. Each
 * sub-world keeps its own contact ids, colouring and overflow list, so its result is bit for
 * bit the result of stepping it as a world of its own. */
int ns_world_begin_subworld(ns_world* world);
int ns_world_subworld_count(const ns_world* world);
/* first_body[count + 1]: the first body id of each sub-world, then the total body count. */
int ns_world_subworld_bodies(const ns_world* world, int* first_body);
/* out[count]: world_state_hash of each sub-world's bodies (synchronises). */
int ns_world_subworld_hashes(ns_world* world, uint64_t* out);

/* Advance one step (replaces World::step solver_integration.rs:807). Asynchronous:
 * the step is enqueued on the world's stream; the first call uploads the scene. dt == 0
 * updates the broadphase pairs only, as the reference does; dt < 0 is NS_ERR_INVALID. */
int ns_world_step(ns_world* world, float dt, int substeps);
/* Adds per-body external force and torque (each n_bodies x 3 floats in body id order, either
 * may be NULL) to the awake bodies for the next step; finalize clears them, as the reference
 * does (replaces apply_body_force_to_center body_api.rs:351 and apply_body_torque :366 for
 * every body at once). The arrays are copied before the call returns. */
int ns_world_apply_forces(ns_world* world, const float* force, const float* torque);
/* Wait for queued steps and report device-side errors (capacity, barrier timeout, non-finite
 * body state). */
int ns_world_synchronize(ns_world* world);

/* Readback (synchronises). Arrays are per body in id order:
 * pos f64x3, rot f32x4 (x,y,z,s), lin f32x3, ang f32x3. Any pointer may be NULL. One device
 * gather packs the state, then each requested array is one copy (pinned host memory makes
 * the copies asynchronous DMA). Reports device errors of the queued steps, like
 * ns_world_synchronize. */
int ns_world_get_bodies(ns_world* world, double* pos, float* rot, float* lin, float* ang);
int ns_world_body_count(const ns_world* world);
/* FNV-1a digest identical to the reference World::world_state_hash (body_queries.rs:432). */
int ns_world_state_hash(ns_world* world, uint64_t* out_hash);
/* Live contacts in id order (same layout as the parity oracle):
 * ints[8] = id, shape a, shape b, color, point count, flags, sat cache type, manifold count;
 * features[4]; floats[24] = normal xyz, then per point anchor_a xyz, separation, normal impulse.
 * Returns the number written (<= capacity) or -1. */
int ns_world_contact_capacity(ns_world* world);
int ns_world_get_contacts(ns_world* world, int32_t* ints, uint32_t* features, float* floats, int capacity);
/* counters[32]: [0] live contacts [1] touching [2..25] per-color constraint counts
 * [26] fast-body flags seen [27] SAT calls (0 on device) [28] recycled contacts last step
 * [29] overflow contacts [30] new pairs last step [31] state changes last step */
int ns_world_counters(ns_world* world, int32_t* counters);

/* Per-step timing of the device phases of the last step, in ms (CUDA events):
 * [0] broadphase [1] collide [2] state pass + color lists + prepare [3] solve [4] finalize. */
int ns_world_phase_times(ns_world* world, float* ms5);
/* Raw CUDA stream (cudaStream_t) the world enqueues on, for callers that time with events. */
void* ns_world_stream(ns_world* world);
/* Solver roofline inputs of the last step (synchronises): [0] awake bodies [1] substeps
 * [2] colored manifolds [3] colored points [4] colored static sides [5] joints
 * [6] overflow contacts [7] restitution on [8] gyroscopic bodies [9] overflow points
 * [10] overflow static sides [11] library kernel launches per step [12] library kernel
 * launches since creation; [13] blocks of the solver launch [14] 1 when that launch is a
 * cooperative grid, 0 when it is one thread-block cluster; [15] dependent phases of the last
 * solver launch (each ends at a barrier over the launch). */
int ns_world_solver_counts(ns_world* world, int64_t* counts16);

/* Batch narrowphase (replaces the per-pair routines collide_hulls_with_scratch
 * convex_manifold.rs:1445, collide_spheres / collide_capsule_and_sphere /
 * collide_capsules / collide_hull_and_sphere / collide_hull_and_capsule
 * convex_manifold_shapes.rs:21-643). Types: 0 capsule, 3 box hull, 5 sphere; A is
 * the primary type (capsule > sphere, hull > sphere/capsule). geom: box hx,hy,hz;
 * sphere cx,cy,cz,r; capsule c1 xyz, c2 xyz, r. xf = B in A's frame (p xyz, q xyzs).
 * The SAT/simplex caches are read and written back. Runs one device thread per pair.
 * Every job is checked on the host before any GPU work, and a batch with one bad job is
 * rejected whole with NS_ERR_INVALID: the pair must be one of the six primary-first pairs
 * above, sat_type 0..8 with sat_hit 0 or 1, a face cache (type 2 or 3) must name a face
 * 0..5, an edge cache (type 4) an even half-edge 0..22 on both boxes, and the simplex cache
 * 0..3 vertices whose indices lie inside the shapes (box 8, capsule 2, sphere 1 vertex). */
typedef struct {
  int32_t type_a, type_b;
  float geom_a[7], geom_b[7];
  float xf[7];
  float sat_separation;
  int32_t sat_type, sat_index_a, sat_index_b, sat_hit;
  float simplex_metric;
  int32_t simplex_count, simplex_ia[4], simplex_ib[4];
} ns_pair_job;
typedef struct {
  float normal[3];
  int32_t point_count;
  float points[4][4]; /* x, y, z, separation in frame A */
  uint32_t feature_ids[4];
} ns_pair_result;
/* Synchronous; host arrays; runs on the calling thread's current CUDA device. */
int ns_collide_pairs(ns_pair_job* jobs, ns_pair_result* results, int count);

/* ns_collide_pairs for callers that must not allocate device memory (no counterpart in the
 * reference). Some hosts cannot call cudaMalloc/cudaFree while they run: an engine whose device
 * memory is fully reserved by its own pool allocator, or a frame loop that may not take the
 * device-wide synchronisation those calls imply. This variant works in a fixed scratch area
 * compiled into the library (about 1 MiB, held on every GPU that loads the library until the
 * process exits) and so handles at most 4096 pairs per call; larger batches are rejected with
 * NS_ERR_CAPACITY before any GPU work (split them into calls of 4096 or fewer). Inputs and
 * outputs are the caller's host arrays, as for ns_collide_pairs, with identical results and
 * the same job checks. The first call on a device sets that device up: it raises the device's
 * per-thread stack limit to what the narrowphase kernel needs (the CUDA driver may allocate the
 * larger local-memory reservation then) and, under lazy module loading, makes the library's
 * module and with it the scratch area resident on the device. That first call may therefore
 * allocate device memory or fail for lack of it: make it once at start-up, before the host's
 * own allocator reserves the device and before any stream capture; later calls allocate
 * nothing. All calls on a device share the one scratch area, so calls that overlap on the GPU
 * (from several host threads, for example) race; serialise them. Runs on the calling thread's
 * current device and returns when the results are in the host arrays. */
int ns_collide_pairs_noalloc(ns_pair_job* jobs, ns_pair_result* results, int count);

/* Diagnostics (no counterpart in the reference): launches the bounded grid barrier of the
 * cooperative solver launch (solver_blocks > 16, or sub-worlds) waiting for one arrival that
 * never comes, so every block gives up after timeout_ms
 * (1..2000). Returns NS_ERR_TIMEOUT when the wait expired and was reported as designed; the
 * CUDA context stays usable afterwards. */
int ns_selftest_barrier_timeout(int device, int timeout_ms);

/* Picks the solver's launch shape for this world by timing (replaces the reference's hand-set
 * CPU worker count, WorldDef::worker_count, src/types/world_def.rs:94): each candidate -- thread-block clusters of 8 and 16 CTAs,
 * cooperative grids over half the SMs and of 1 to 4 blocks per SM as far as they fit -- steps the world
 * for 1 + steps steps of (dt, substeps) from a copy of its current state, timed with CUDA events;
 * the fastest is kept and the world is put back exactly as it was (every shape gives the same
 * bits). Per candidate c < max_candidates: blocks_out[c], grid_out[c] (1 cooperative grid, 0
 * cluster) and ms_out[c] (ms per step, -1 for a cluster that does not fit); any may be NULL.
 * Returns the number of candidates (>= 1), or minus an NS_ERR_* status (message in
 * ns_last_error). Refused while a tape records. */
int ns_world_autotune(ns_world* w, float dt, int substeps, int steps, int* blocks_out, int* grid_out,
                      float* ms_out, int max_candidates);
/* After the solver's shape, ns_world_autotune tunes, one kernel at a time from the same copy of
 * the world, the launch shapes of the narrowphase recycle pass (contacts per thread: threads per
 * block and blocks per SM), the full manifold updates and the constraint preparation, and keeps
 * the fastest of each (every shape gives the same bits). ns_world_autotune_table lists every
 * timed candidate of the last call: dimension (0 solver, 1 recycle pass, 2 manifold updates,
 * 3 preparation), value_a (blocks of the solver launch, or threads per block), value_b (1 for a
 * cooperative solver grid / 0 for a cluster, or blocks per SM at most) and ms per step (-1 when
 * a cluster size does not fit). Returns the number of rows (any output may be NULL). */
int ns_world_autotune_table(const ns_world* w, int* dimension, int* value_a, int* value_b, float* ms,
                            int max_rows);
/* out8: solver blocks, cooperative grid (0/1), recycle threads per block, recycle blocks per SM,
 * update threads, update blocks per SM, prepare threads, prepare blocks per SM. */
int ns_world_launch_shapes(const ns_world* w, int* out8);
/* Sets the launch shapes (the same 8 values) directly, e.g. ones an earlier autotune chose on a
 * world of the same kind at a representative step. Threads per block must be multiples of 32
 * within each kernel's launch bound (256, 64, 128), blocks per SM 1..64, a cluster 1..16 CTAs
 * that fits, a cooperative grid co-resident; NS_ERR_INVALID otherwise. Uploads the scene if it
 * is not yet on the device. Every shape gives the same bits. */
int ns_world_set_launch_shapes(ns_world* w, const int* in8);

/* ---- Adjoint: vector-Jacobian product of a recorded rollout --------------------------------
 * No counterpart in the reference, which has no differentiation; these calls are the
 * differentiable form of World::step (solver_integration.rs:807) built on the same step.
 *
 * ns_world_tape_begin starts recording: every later ns_world_step is logged, and the world's
 * device state is copied to a checkpoint at the start and whenever checkpoint_substeps
 * substeps have passed since the last checkpoint (steps are whole, so a checkpoint falls on
 * the first step boundary at or after that count). While recording, dt must be > 0 and
 * ns_world_apply_forces is refused. Scope: one world (no sub-worlds) of box, sphere and
 * capsule bodies with the centre of mass at the body origin and revolute joints (none in the
 * overflow colour), without kinematic bodies, rolling resistance or continuous collision
 * (NS_ERR_UNSUPPORTED otherwise); steps that put contacts in the overflow colour are reported
 * by ns_world_vjp as NS_ERR_UNSUPPORTED, and steps with restitution, or worlds with joints, by
 * ns_world_vjp_f64. */
int ns_world_tape_begin(ns_world* w, int checkpoint_substeps);
/* Stops recording; the tape stays for ns_world_vjp. */
int ns_world_tape_end(ns_world* w);
/* Releases the tape and its checkpoints. The checkpoints' device memory (and the VJP's scratch)
 * stays with the world for the next tape, so repeated rollouts allocate nothing after the first;
 * ns_world_destroy frees it. */
int ns_world_tape_free(ns_world* w);
/* out[8]: recorded steps, checkpoints, narrowphase replays that did not reproduce the
 * recorded manifold (their pose derivatives are left out), VJP calls, recording (0/1),
 * checkpoint interval in substeps, own kernel launches of the last VJP, 0. */
int ns_world_tape_info(ns_world* w, int64_t* out);
/* Cotangents of the world's state after the last recorded step, in body id order (rows as
 * ns_world_get_bodies: position xyz, rotation xyzw, linear and angular velocity; any may be
 * NULL for zero), are pulled back to the state and parameters at ns_world_tape_begin:
 * initial linear and angular velocity (3 per body), body mass (the density scale: inverse
 * mass and inverse inertia scale as 1/m, inertia as m), the friction of the body's shape, initial position
 * (3) and rotation (4). Any output may be NULL; static bodies get zeros. The recorded steps
 * are replayed from the checkpoints (bit-identical to the recorded run) to rebuild the
 * intermediate state, and the world is left in its state after the last recorded step.
 * Gradients are exact for the branch the rollout took (contact sets, clamps and friction
 * cones are held). Synchronous. */
int ns_world_vjp(ns_world* w, const float* dpos, const float* drot, const float* dlin, const float* dang,
                 float* dlin0, float* dang0, float* dmass, float* dfriction, float* dpos0, float* drot0);
/* drestitution[n_bodies]: the last ns_world_vjp's cotangent of each body's shape restitution
 * (a contact's coefficient is the larger of its two shapes', world_runtime.rs mix_restitution,
 * and its cotangent goes to the body whose shape supplied it; zero for bodies no restitution
 * update reached). NS_ERR_INVALID before the first ns_world_vjp or after bodies were added. */
int ns_world_vjp_restitution(const ns_world* w, float* drestitution);
/* The same vector-Jacobian product with the reverse pass run on the host in f64 (the replay of
 * the recorded steps still runs on the GPU, bit-identical to the recording): the f64 reference
 * for ns_world_vjp's f32 device pass. Same arguments, outputs in double; much slower (one CPU
 * thread). No counterpart in the reference. */
int ns_world_vjp_f64(ns_world* w, const float* dpos, const float* drot, const float* dlin, const float* dang,
                     double* dlin0, double* dang0, double* dmass, double* dfriction, double* dpos0, double* drot0);

/* Diagnostics (no counterpart in the reference): an f64 check, on the host without a GPU, of
 * one local derivative the adjoint uses (which: 0 warm start, 1 push, 2 relax, 3 prepare,
 * 4 integrate velocities, 5 integrate positions, 6 finalize rotation, 7 inverse world inertia,
 * 8 recycled separations, 9..11 box-box manifolds: face, any axis, edge pair) at seeded random
 * inputs. worst[0] = the largest relative difference between the dual-number vector-Jacobian
 * product and central differences over all input directions; worst[1] = the separating-axis
 * kind of the box cases (-1 otherwise). which 12..16 instead compare the hand-written reverse
 * sweeps the GPU runs for warm start, push, relax (also their state-and-impulse-only form),
 * integrate positions and integrate velocities (without the gyroscopic step) with the
 * dual-number products. which 17 checks restitution like 0..11; which 18 compares the
 * hand-written reverse of the relative normal velocity prepare samples with the dual numbers.
 * which 19..23 check the manifolds of sphere-sphere, capsule-sphere, capsule-capsule,
 * box-sphere and box-capsule pairs like 9..11; worst[1] = the point count (19..21) or the
 * replayed path (22, 23: 2 GJK point, 3 GJK face, 4 face, 5 edge pair). which 24..26 check the
 * revolute joint's solve, warm start and prepare like 0..8. */
int ns_adjoint_selfcheck(int which, int seed, double* worst);

#ifdef __cplusplus
}
#endif
#endif
