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
  int enable_continuous;     /* 1 = flag fast bodies (CCD itself is out of scope) */
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
void nso_step(nso_world* w, float dt, int substeps);
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

#ifdef __cplusplus
}
#endif
#endif
