/* Oracle C interface. TEST INFRASTRUCTURE ONLY: the CPU restatement of the
 * reference's scalar world step, used by tests/, __graft_entry__.smoke() and
 * bench.py's CPU baseline as the parity checker. The product library never
 * links it. Scene-building calls mirror the reference's World API
 * (simulation/world_runtime.rs:1506 create_body, shape_creation.rs:504-569,
 * joint.rs:164) so the same seeded scene can be built in both libraries. */
#ifndef NS_ORACLE_H
#define NS_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct nso_world nso_world;

typedef struct {
  float gravity[3];
  int enable_sleep;          /* must be 0: sleeping islands are out of scope */
  int enable_continuous;     /* 1 = continuous pass of fast bodies against static shapes */
  int enable_warm_starting;
  float contact_hertz;
  float contact_damping_ratio;
  float contact_speed;
  float max_linear_speed;
  float restitution_threshold;
  int restitution_iterations;
  float joint_hertz;
  float joint_damping_ratio;
} nso_world_def;

typedef struct {
  int type; /* 0 static, 2 dynamic */
  double position[3];
  float rotation[4]; /* x, y, z, s */
  float linear_velocity[3];
  float angular_velocity[3];
  float linear_damping, angular_damping, gravity_scale;
  int enable_sleep;
  int is_bullet;
} nso_body_def;

typedef struct {
  float density, friction, restitution, rolling_resistance;
  uint64_t category_bits, mask_bits;
  int group_index;
} nso_shape_def;

void nso_default_world_def(nso_world_def* def);
nso_world* nso_create(const nso_world_def* def);
void nso_destroy(nso_world* w);
int nso_create_body(nso_world* w, const nso_body_def* def);
int nso_create_box(nso_world* w, int body, const nso_shape_def* def, float hx, float hy, float hz);
int nso_create_sphere(nso_world* w, int body, const nso_shape_def* def, const float center[3], float radius);
int nso_create_capsule(nso_world* w, int body, const nso_shape_def* def, const float c1[3],
                       const float c2[3], float radius);
/* Revolute joint: frames are local to the body origins (position + rotation xyzs). */
int nso_create_revolute(nso_world* w, int body_a, int body_b, const float frame_a[7],
                        const float frame_b[7], int enable_limit, float lower, float upper,
                        int enable_spring, float hertz, float damping_ratio, float drag_torque,
                        int collide_connected);
/* The whole RevoluteJointDef (types/joint_defs.rs:154 with its JointDef base :30); same layout
 * as the product's ns_revolute_joint_def. */
typedef struct {
  int body_a, body_b;
  float local_frame_a[7], local_frame_b[7];
  float constraint_hertz, constraint_damping_ratio;
  int collide_connected;
  float target_angle;
  int enable_spring;
  float hertz, damping_ratio;
  int enable_limit;
  float lower_angle, upper_angle;
  int enable_motor;
  float max_motor_torque, motor_speed;
} nso_revolute_def;
int nso_create_revolute_def(nso_world* w, const nso_revolute_def* def);
/* SphericalJointDef (types/joint_defs.rs:169 with its JointDef base :30); same layout as the
 * product's ns_spherical_joint_def. */
typedef struct {
  int body_a, body_b;
  float local_frame_a[7], local_frame_b[7];
  float constraint_hertz, constraint_damping_ratio;
  int collide_connected;
  int enable_spring;
  float hertz, damping_ratio;
  float target_rotation[4];
  int enable_cone_limit;
  float cone_angle;
  int enable_twist_limit;
  float lower_twist_angle, upper_twist_angle;
  int enable_motor;
  float max_motor_torque;
  float motor_velocity[3];
} nso_spherical_def;
int nso_create_spherical_def(nso_world* w, const nso_spherical_def* def);
void nso_step(nso_world* w, float dt, int substeps);
/* Host threads of the colour-parallel loops (all worlds of the process; default 1). */
void nso_set_threads(int threads);
/* Per-body force / torque (n_bodies x 3, id order, either may be NULL) for the next step. */
void nso_apply_forces(nso_world* w, const float* force, const float* torque);
uint64_t nso_state_hash(const nso_world* w);
int nso_body_count(const nso_world* w);
/* Per body (id order): position f64x3, rotation f32x4, linear/angular velocity f32x3 each. */
int nso_get_bodies(const nso_world* w, double* pos, float* rot, float* lin, float* ang);
/* Live contacts in id order: id, shape a, shape b, color, point count, flags; feature ids (4),
 * normal (3), per point anchor a (3), separation, normal impulse (4 points x 5). */
int nso_contact_capacity(const nso_world* w);
int nso_get_contacts(const nso_world* w, int32_t* ints /* cap*8 */, uint32_t* features /* cap*4 */,
                     float* floats /* cap*24 */);
/* counters: [0]=live contacts [1]=touching [2..25]=color counts [26]=fast-body flags seen
 * [27]=sat calls [28]=recycled last step */
void nso_counters(const nso_world* w, int32_t* out /* 32 */);

/* One narrowphase pair (collision/convex_manifold*.rs entry points). Types: 0 capsule,
 * 3 box hull, 5 sphere; A must be the primary type (capsule>sphere, hull>sphere/capsule).
 * geom: box hx,hy,hz; sphere cx,cy,cz,r; capsule c1 xyz, c2 xyz, r. xf = B in A's frame
 * (p xyz, q xyzs). The caches are read and written back. */
typedef struct {
  int32_t type_a, type_b;
  float geom_a[7], geom_b[7];
  float xf[7];
  float sat_separation;
  int32_t sat_type, sat_index_a, sat_index_b, sat_hit;
  float simplex_metric;
  int32_t simplex_count, simplex_ia[4], simplex_ib[4];
} nso_pair_job;
typedef struct {
  float normal[3];
  int32_t point_count;
  float points[4][4]; /* x, y, z, separation (frame A) */
  uint32_t feature_ids[4];
} nso_pair_result;
void nso_collide_pairs(nso_pair_job* jobs, nso_pair_result* results, int count);

/* One time-of-impact query (collision/time_of_impact.rs:391). Proxies: up to 8 points (xyz) and
 * a radius. Sweeps: local_center xyz, c1 xyz, c2 xyz, q1 xyzs, q2 xyzs (17 floats).
 * out[13]: state (0 unknown, 1 failed, 2 overlapped, 3 hit, 4 separated), fraction, distance,
 * point xyz, normal xyz, distance / push-back / root iterations. */
void nso_time_of_impact(const float* points_a, int count_a, float radius_a, const float* points_b, int count_b,
                        float radius_b, const float* sweep_a, const float* sweep_b, float max_fraction, float* out);

#ifdef __cplusplus
}
#endif
#endif
