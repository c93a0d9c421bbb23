// Oracle joint rows. TEST INFRASTRUCTURE ONLY (the parity checker).
// Restates simulation/revolute_joint.rs, simulation/spherical_joint.rs and the joint dispatch of
// simulation/distance_joint_solver.rs:74-346 for those two types.
#pragma once
#include <vector>
#include "ns_math.hpp"

namespace nso {

struct JointSoft { real bias_rate, mass_scale, impulse_scale; };

inline JointSoft joint_make_soft(real hertz, real zeta, real h) {  // solver_integration.rs:72
  JointSoft s = {0, 0, 0};
  if (hertz == 0.0f) return s;
  real omega = 2.0f * kPi * hertz;
  real a1 = 2.0f * zeta + h * omega;
  real a2 = h * omega * a1;
  real a3 = 1.0f / (1.0f + a2);
  s.bias_rate = omega / a1;
  s.mass_scale = a2 * a3;
  s.impulse_scale = a3;
  return s;
}

struct Joint {
  int id = -1, body_a = -1, body_b = -1, color = -1;
  bool collide_connected = false;
  Xf local_frame_a, local_frame_b;
  real constraint_hertz = 60.0f, constraint_damping_ratio = 2.0f;
  JointSoft constraint_softness = {0.0f, 1.0f, 0.0f};
  real inv_mass_a = 0, inv_mass_b = 0;
  M3 inv_ia, inv_ib;
  bool fixed_rotation = false;
  // RevoluteJointSim (revolute_joint.rs:28)
  V3 linear_impulse = {0, 0, 0};
  V2 perp_impulse = {0, 0};
  real spring_impulse = 0, motor_impulse = 0, lower_impulse = 0, upper_impulse = 0;
  real hertz = 0, damping_ratio = 0, max_motor_torque = 0, motor_speed = 0, target_angle = 0;
  real lower_angle = 0, upper_angle = 0;
  int index_a = -1, index_b = -1;
  Xf frame_a, frame_b;
  V3 rotation_axis_z, perp_axis_x, perp_axis_y, delta_center;
  real axial_mass = 0;
  JointSoft spring_softness = {0, 0, 0};
  bool enable_spring = false, enable_motor = false, enable_limit = false;
  // SphericalJointSim (spherical_joint.rs:40): type 1. lower_impulse / upper_impulse hold the
  // twist limit impulses; the spring and motor impulses are vectors.
  int type = 0;
  bool enable_cone_limit = false, enable_twist_limit = false;
  real cone_angle = 0, lower_twist_angle = 0, upper_twist_angle = 0;
  Q target_rotation = {{0, 0, 0}, 1};
  V3 motor_velocity = {0, 0, 0}, spring_impulse3 = {0, 0, 0}, motor_impulse3 = {0, 0, 0};
  real swing_impulse = 0, swing_mass = 0, twist_mass = 0;
  V3 swing_axis = {0, 0, 0}, twist_jacobian = {0, 0, 0};
  M3 rotation_mass = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
};

// spherical_joint.rs:119 create_spherical_joint
inline Joint make_spherical_joint(int a, int b, const float* fa, const float* fb, bool collide, real c_hertz,
                                  real c_zeta, bool spring, real hertz, real zeta, Q target, bool cone,
                                  real cone_angle, bool twist, real lower, real upper, bool motor,
                                  real max_torque, V3 motor_velocity) {
  Joint j;
  j.type = 1;
  j.body_a = a; j.body_b = b;
  j.local_frame_a = xf(v3(fa[0], fa[1], fa[2]), quat(v3(fa[3], fa[4], fa[5]), fa[6]));
  j.local_frame_b = xf(v3(fb[0], fb[1], fb[2]), quat(v3(fb[3], fb[4], fb[5]), fb[6]));
  j.collide_connected = collide;
  j.constraint_hertz = c_hertz; j.constraint_damping_ratio = c_zeta;
  j.enable_spring = spring; j.hertz = hertz; j.damping_ratio = zeta; j.target_rotation = target;
  j.enable_cone_limit = cone; j.cone_angle = cone_angle;
  j.enable_twist_limit = twist; j.lower_twist_angle = lower; j.upper_twist_angle = upper;
  j.enable_motor = motor; j.max_motor_torque = max_torque; j.motor_velocity = motor_velocity;
  j.inv_ia = m3zero(); j.inv_ib = m3zero();
  return j;
}

// internal_math.rs:328 delta_quat_to_rotation
inline V3 delta_quat_to_rotation(Q q, Q target) {
  Q s = dot_quat(q, target) < 0.0f ? quat(v3(-q.v.x, -q.v.y, -q.v.z), -q.s) : q;
  Q diff = quat(target.v - s.v, target.s - s.s);
  Q product = mul_quat(diff, conjugate(s));
  return 2.0f * product.v;
}
// functions.rs:502 get_swing_angle
inline real get_swing_angle(Q q) {
  real x = std::sqrt(q.v.z * q.v.z + q.s * q.s);
  real y = std::sqrt(q.v.x * q.v.x + q.v.y * q.v.y);
  return 2.0f * atan2_approx(y, x);
}

inline Joint make_revolute_joint(int a, int b, const float* fa, const float* fb, bool limit, real lower,
                                 real upper, bool spring, real hertz, real zeta, real drag,
                                 bool collide, real c_hertz, real c_zeta) {
  Joint j;
  j.body_a = a; j.body_b = b;
  j.local_frame_a = xf(v3(fa[0], fa[1], fa[2]), quat(v3(fa[3], fa[4], fa[5]), fa[6]));
  j.local_frame_b = xf(v3(fb[0], fb[1], fb[2]), quat(v3(fb[3], fb[4], fb[5]), fb[6]));
  j.enable_limit = limit; j.lower_angle = lower; j.upper_angle = upper;
  j.enable_spring = spring; j.hertz = hertz; j.damping_ratio = zeta;
  j.max_motor_torque = drag;
  j.enable_motor = drag > 0.0f;
  j.collide_connected = collide;
  j.constraint_hertz = c_hertz; j.constraint_damping_ratio = c_zeta;
  j.inv_ia = m3zero(); j.inv_ib = m3zero();
  return j;
}

// revolute_joint.rs:95 solve_point_constraint
inline V3 solve_point_constraint(real ma, real mb, M3 ia, M3 ib, V3 ra, V3 rb, V3 rhs) {
  real axy = ra.z * ia.cy.y - ra.y * ia.cz.y;
  real axz = ra.z * ia.cy.z - ra.y * ia.cz.z;
  V3 ay = ra.x * ia.cz - ra.z * ia.cx;
  V3 az = ra.y * ia.cx - ra.x * ia.cy;
  real bxy = rb.z * ib.cy.y - rb.y * ib.cz.y;
  real bxz = rb.z * ib.cy.z - rb.y * ib.cz.z;
  V3 by = rb.x * ib.cz - rb.z * ib.cx;
  V3 bz = rb.y * ib.cx - rb.x * ib.cy;
  real m = ma + mb;
  real kxx = (axy * ra.z - axz * ra.y) + (bxy * rb.z - bxz * rb.y) + m;
  real kyy = (ay.z * ra.x - ay.x * ra.z) + (by.z * rb.x - by.x * rb.z) + m;
  real kzz = (az.x * ra.y - az.y * ra.x) + (bz.x * rb.y - bz.y * rb.x) + m;
  real kxy = (ay.y * ra.z - ay.z * ra.y) + (by.y * rb.z - by.z * rb.y);
  real kxz = (az.y * ra.z - az.z * ra.y) + (bz.y * rb.z - bz.z * rb.y);
  real kyz = (az.z * ra.x - az.x * ra.z) + (bz.z * rb.x - bz.x * rb.z);
  real cxx = kyy * kzz - kyz * kyz;
  real cyy = kxx * kzz - kxz * kxz;
  real czz = kxx * kyy - kxy * kxy;
  real cxy = kxz * kyz - kxy * kzz;
  real cxz = kxy * kyz - kyy * kxz;
  real cyz = kxy * kxz - kxx * kyz;
  real d = kxx * cxx + kxy * cxy + kxz * cxz;
  if (absf(d) > 1000.0f * kMinPositive) {
    real inv = 1.0f / d;
    return v3(inv * (cxx * rhs.x + cxy * rhs.y + cxz * rhs.z),
              inv * (cxy * rhs.x + cyy * rhs.y + cyz * rhs.z),
              inv * (cxz * rhs.x + cyz * rhs.y + czz * rhs.z));
  }
  return v3(0, 0, 0);
}

}  // namespace nso

// The joint stage functions need the world's body arrays; they are templates so this header
// does not depend on the world's private types.
namespace nso {

// spherical_joint.rs:183-230: the spherical joint's part of prepare (after the common frames)
inline void prepare_spherical(Joint& j, M3 inv_inertia_sum, real h, real warm) {
  V3 cone_axis = rotate(j.frame_a.q, v3(0, 0, 1));
  V3 twist_axis = rotate(j.frame_b.q, v3(0, 0, 1));
  if (j.enable_cone_limit) {
    V3 swing_axis = normalize(cross(cone_axis, twist_axis));
    real k = dot(swing_axis, mul_mv(inv_inertia_sum, swing_axis));
    j.swing_mass = k > 0.0f ? 1.0f / k : 0.0f;
    j.swing_axis = swing_axis;
  }
  if (j.enable_twist_limit) {
    Q rel_q = inv_mul_quat(j.frame_a.q, j.frame_b.q);
    real tan_half = std::sqrt((rel_q.v.x * rel_q.v.x + rel_q.v.y * rel_q.v.y) /
                              (rel_q.v.z * rel_q.v.z + rel_q.s * rel_q.s));
    V3 swing_axis = normalize(cross(cone_axis, twist_axis));
    V3 perp_axis = cross(swing_axis, cone_axis);
    V3 jac = mul_add(cone_axis, tan_half, perp_axis);
    real k = dot(jac, mul_mv(inv_inertia_sum, jac));
    j.twist_mass = k > 0.0f ? 1.0f / k : 0.0f;
    j.twist_jacobian = jac;
  }
  j.rotation_mass = !j.fixed_rotation ? invert_matrix(inv_inertia_sum) : m3zero();
  j.spring_softness = joint_make_soft(j.hertz, j.damping_ratio, h);
  if (warm == 0.0f) {
    j.linear_impulse = v3(0, 0, 0); j.motor_impulse3 = v3(0, 0, 0); j.spring_impulse3 = v3(0, 0, 0);
    j.swing_impulse = 0; j.lower_impulse = 0; j.upper_impulse = 0;
  }
}

template <class BodyT, class SimT>
void prepare_joints(std::vector<Joint>& joints, const std::vector<SimT>& awake, const std::vector<SimT>& stat,
                    const BodyT* bodies, real h, real inv_h, real warm) {
  for (Joint& j : joints) {
    // distance_joint_solver.rs:74 prepare_joint
    real hz = minf(j.constraint_hertz, 0.25f * inv_h);
    j.constraint_softness = joint_make_soft(hz, j.constraint_damping_ratio, h);
    // revolute_joint.rs:183 prepare_revolute_joint
    const BodyT& ba = bodies[j.body_a];
    const BodyT& bb = bodies[j.body_b];
    const SimT& sa = ba.set_index == 2 ? awake[ba.local_index] : stat[ba.local_index];
    const SimT& sb = bb.set_index == 2 ? awake[bb.local_index] : stat[bb.local_index];
    j.inv_mass_a = sa.inv_mass; j.inv_mass_b = sb.inv_mass;
    j.inv_ia = sa.inv_inertia_world; j.inv_ib = sb.inv_inertia_world;
    M3 sum = add_mm(j.inv_ia, j.inv_ib);
    j.fixed_rotation = det(sum) < 1000.0f * kMinPositive;
    j.index_a = ba.set_index == 2 ? ba.local_index : -1;
    j.index_b = bb.set_index == 2 ? bb.local_index : -1;
    j.frame_a.q = mul_quat(sa.transform.q, j.local_frame_a.q);
    j.frame_a.p = rotate(sa.transform.q, j.local_frame_a.p - sa.local_center);
    j.frame_b.q = mul_quat(sb.transform.q, j.local_frame_b.q);
    j.frame_b.p = rotate(sb.transform.q, j.local_frame_b.p - sb.local_center);
    j.delta_center = sub_pos(sb.center, sa.center);
    if (j.type == 1) {
      prepare_spherical(j, sum, h, warm);
      continue;
    }
    V3 axis = rotate(j.frame_a.q, v3(0, 0, 1));
    real k = dot(axis, mul_mv(sum, axis));
    j.axial_mass = k > 0.0f ? 1.0f / k : 0.0f;
    j.rotation_axis_z = axis;
    Q rq = inv_mul_quat(j.frame_a.q, j.frame_b.q);
    j.perp_axis_x = 0.5f * rotate(j.frame_a.q, rq.s * v3(1, 0, 0) + cross(rq.v, v3(1, 0, 0)));
    j.perp_axis_y = 0.5f * rotate(j.frame_a.q, rq.s * v3(0, 1, 0) + cross(rq.v, v3(0, 1, 0)));
    j.spring_softness = joint_make_soft(j.hertz, j.damping_ratio, h);
    if (warm == 0.0f) {
      j.linear_impulse = v3(0, 0, 0); j.perp_impulse = v2(0, 0);
      j.motor_impulse = 0; j.spring_impulse = 0; j.lower_impulse = 0; j.upper_impulse = 0;
    }
  }
}

template <class StateT>
StateT joint_state_at(std::vector<StateT>& states, int i) {
  if (i >= 0) return states[i];
  StateT s;
  s.v = v3(0, 0, 0); s.w = v3(0, 0, 0); s.dp = v3(0, 0, 0); s.flags = 0; s.dq = qid();
  return s;
}

// spherical_joint.rs:315-438: the spring, motor, twist limit and cone limit rows of
// solve_spherical_joint (the point constraint is shared with the revolute joint)
inline void solve_spherical_angular(Joint& j, Q qa, Q qb, M3 iA, M3 iB, real h, real inv_h, bool use_bias, V3& wa,
                                    V3& wb) {
  Q rel_q = inv_mul_quat(qa, qb);
  if (j.fixed_rotation || !(j.enable_spring || j.enable_motor || j.enable_twist_limit || j.enable_cone_limit)) return;
  M3 sum = add_mm(iA, iB);
  V3 cdot = wb - wa;
  V3 ang = v3(0, 0, 0);
  if (j.enable_spring) {
    V3 dr = delta_quat_to_rotation(rel_q, j.target_rotation);
    V3 c = -(rotate(qa, dr));
    V3 bias = j.spring_softness.bias_rate * c;
    real ms = j.spring_softness.mass_scale, is = j.spring_softness.impulse_scale;
    V3 imp = (-ms) * mul_mv(j.rotation_mass, cdot + bias) - is * j.spring_impulse3;
    j.spring_impulse3 = j.spring_impulse3 + imp;
    cdot = cdot + mul_mv(sum, imp);
    ang = ang + imp;
  }
  if (j.enable_motor) {
    V3 lambda = -(mul_mv(j.rotation_mass, cdot - j.motor_velocity));
    V3 next = j.motor_impulse3 + lambda;
    real len = length(next);
    real mx = j.max_motor_torque * h;
    if (len > mx) next = (mx / len) * next;
    lambda = next - j.motor_impulse3;
    j.motor_impulse3 = next;
    cdot = cdot + mul_mv(sum, lambda);
    ang = ang + lambda;
  }
  auto limit_terms = [&](real c, real& bias, real& ms, real& is) {
    bias = 0.0f; ms = 1.0f; is = 0.0f;
    if (c > 0.0f) bias = c * inv_h;
    else if (use_bias) {
      bias = j.constraint_softness.bias_rate * c;
      ms = j.constraint_softness.mass_scale;
      is = j.constraint_softness.impulse_scale;
    }
  };
  if (j.enable_twist_limit) {
    real twist = get_twist_angle(rel_q);
    V3 jac = j.twist_jacobian;
    V3 resp = mul_mv(sum, jac);
    {
      real bias, ms, is;
      limit_terms(twist - j.lower_twist_angle, bias, ms, is);
      real tcd = dot(cdot, jac);
      real old = j.lower_impulse;
      real di = maxf(-ms * j.twist_mass * (tcd + bias) - is * old, -old);
      j.lower_impulse = old + di;
      cdot = mul_add(cdot, di, resp);
      ang = mul_add(ang, di, jac);
    }
    {
      real bias, ms, is;
      limit_terms(j.upper_twist_angle - twist, bias, ms, is);
      real tcd = -dot(cdot, jac);
      real old = j.upper_impulse;
      real di = maxf(-ms * j.twist_mass * (tcd + bias) - is * old, -old);
      j.upper_impulse = old + di;
      cdot = cdot - di * resp;
      ang = ang - di * jac;
    }
  }
  if (j.enable_cone_limit) {
    real swing = get_swing_angle(rel_q);
    real bias, ms, is;
    limit_terms(j.cone_angle - swing, bias, ms, is);
    real scd = -dot(cdot, j.swing_axis);
    real old = j.swing_impulse;
    real di = maxf(-ms * j.swing_mass * (scd + bias) - is * old, -old);
    j.swing_impulse = old + di;
    ang = ang - di * j.swing_axis;
  }
  wa = wa - mul_mv(iA, ang);
  wb = wb + mul_mv(iB, ang);
}

// revolute_joint.rs:261 warm_start_revolute_joint
template <class StateT>
void warm_start_joints_color(std::vector<Joint>& joints, const std::vector<int>& ids,
                             std::vector<StateT>& states, real h) {
  (void)h;
  for (int id : ids) {
    Joint& j = joints[id];
    real mA = j.inv_mass_a, mB = j.inv_mass_b;
    StateT sa = joint_state_at(states, j.index_a), sb = joint_state_at(states, j.index_b);
    V3 va = sa.v, wa = sa.w, vb = sb.v, wb = sb.w;
    V3 ra = rotate(sa.dq, j.frame_a.p), rb = rotate(sb.dq, j.frame_b.p);
    V3 ang;
    if (j.type == 1) {  // spherical_joint.rs:233 warm_start_spherical_joint
      ang = j.spring_impulse3 + j.motor_impulse3;
      ang = ang - j.swing_impulse * j.swing_axis;
      ang = mul_add(ang, j.lower_impulse - j.upper_impulse, j.twist_jacobian);
    } else {
      real axial = j.spring_impulse + j.motor_impulse + j.lower_impulse - j.upper_impulse;
      ang = j.perp_impulse.x * j.perp_axis_x + j.perp_impulse.y * j.perp_axis_y;
      ang = mul_add(ang, axial, j.rotation_axis_z);
    }
    va = va - mA * j.linear_impulse;
    wa = wa - mul_mv(j.inv_ia, cross(ra, j.linear_impulse) + ang);
    vb = vb + mB * j.linear_impulse;
    wb = wb + mul_mv(j.inv_ib, cross(rb, j.linear_impulse) + ang);
    if (sa.flags & 0x1000u) { sa.v = va; sa.w = wa; }
    if (sb.flags & 0x1000u) { sb.v = vb; sb.w = wb; }
    if (j.index_a >= 0 && (sa.flags & 0x1000u)) states[j.index_a] = sa;
    if (j.index_b >= 0 && (sb.flags & 0x1000u)) states[j.index_b] = sb;
  }
}

// revolute_joint.rs:316 solve_revolute_joint
template <class StateT>
void solve_joints_color(std::vector<Joint>& joints, const std::vector<int>& ids, std::vector<StateT>& states,
                        real h, real inv_h, bool use_bias) {
  for (int id : ids) {
    Joint& j = joints[id];
    real mA = j.inv_mass_a, mB = j.inv_mass_b;
    M3 iA = j.inv_ia, iB = j.inv_ib;
    StateT sa = joint_state_at(states, j.index_a), sb = joint_state_at(states, j.index_b);
    V3 va = sa.v, wa = sa.w, vb = sb.v, wb = sb.w;
    bool fixed = j.fixed_rotation;
    Q qa = mul_quat(sa.dq, j.frame_a.q);
    Q qb = mul_quat(sb.dq, j.frame_b.q);
    if (j.type == 1) {
      solve_spherical_angular(j, qa, qb, iA, iB, h, inv_h, use_bias, wa, wb);
    } else {
    if (dot_quat(qa, qb) < 0.0f) qb = quat(v3(-qb.v.x, -qb.v.y, -qb.v.z), -qb.s);
    Q rq = inv_mul_quat(qa, qb);
    if (!fixed && (j.enable_spring || j.enable_motor || j.enable_limit)) {
      V3 axis = j.rotation_axis_z;
      V3 ga = mul_mv(iA, axis), gb = mul_mv(iB, axis);
      real k = dot(axis, ga + gb);
      real acd = dot(wb - wa, axis);
      real ai = 0.0f;
      if (j.enable_spring) {
        real angle = get_twist_angle(rq);
        real c = angle - j.target_angle;
        real bias = j.spring_softness.bias_rate * c;
        real ms = j.spring_softness.mass_scale, is = j.spring_softness.impulse_scale;
        real di = -ms * j.axial_mass * (acd + bias) - is * j.spring_impulse;
        j.spring_impulse += di;
        acd += k * di;
        ai += di;
      }
      if (j.enable_motor) {
        real cdot = acd - j.motor_speed;
        real old = j.motor_impulse;
        real mx = j.max_motor_torque * h;
        real di = clampf(-j.axial_mass * cdot, -mx - old, mx - old);
        j.motor_impulse = old + di;
        acd += k * di;
        ai += di;
      }
      if (j.enable_limit) {
        real angle = get_twist_angle(rq);
        {
          real c = angle - j.lower_angle;
          real bias = 0.0f, ms = 1.0f, is = 0.0f;
          if (c > 0.0f) bias = c * inv_h;
          else if (use_bias) {
            bias = j.constraint_softness.bias_rate * c;
            ms = j.constraint_softness.mass_scale;
            is = j.constraint_softness.impulse_scale;
          }
          real old = j.lower_impulse;
          real di = maxf(-ms * j.axial_mass * (acd + bias) - is * old, -old);
          j.lower_impulse = old + di;
          acd += k * di;
          ai += di;
        }
        {
          real c = j.upper_angle - angle;
          real bias = 0.0f, ms = 1.0f, is = 0.0f;
          if (c > 0.0f) bias = c * inv_h;
          else if (use_bias) {
            bias = j.constraint_softness.bias_rate * c;
            ms = j.constraint_softness.mass_scale;
            is = j.constraint_softness.impulse_scale;
          }
          real cdot = -acd;
          real old = j.upper_impulse;
          real di = maxf(-ms * j.axial_mass * (cdot + bias) - is * old, -old);
          j.upper_impulse = old + di;
          ai -= di;
        }
      }
      wa = wa - ai * ga;
      wb = wb + ai * gb;
    }
    if (!fixed) {
      V2 bias = v2(0, 0);
      real ms = 1.0f, is = 0.0f;
      if (use_bias) {
        V2 c = v2(rq.v.x, rq.v.y);
        bias = v2(j.constraint_softness.bias_rate * c.x, j.constraint_softness.bias_rate * c.y);
        ms = j.constraint_softness.mass_scale;
        is = j.constraint_softness.impulse_scale;
      }
      V3 px = 0.5f * rotate(qa, rq.s * v3(1, 0, 0) + cross(rq.v, v3(1, 0, 0)));
      V3 py = 0.5f * rotate(qa, rq.s * v3(0, 1, 0) + cross(rq.v, v3(0, 1, 0)));
      j.perp_axis_x = px;
      j.perp_axis_y = py;
      M3 sum = add_mm(iA, iB);
      real kxx = dot(px, mul_mv(sum, px));
      real kyy = dot(py, mul_mv(sum, py));
      real kxy = dot(px, mul_mv(sum, py));
      M2 K;
      K.cx = v2(kxx, kxy);
      K.cy = v2(kxy, kyy);
      V3 wr = wb - wa;
      V2 cdot = v2(dot(wr, px), dot(wr, py));
      V2 old = j.perp_impulse;
      V2 sol = solve2(K, v2(cdot.x + bias.x, cdot.y + bias.y));
      V2 di = v2((-ms) * sol.x - is * old.x, (-ms) * sol.y - is * old.y);
      j.perp_impulse = v2(j.perp_impulse.x + di.x, j.perp_impulse.y + di.y);
      V3 ang = di.x * px + di.y * py;
      wa = wa - mul_mv(iA, ang);
      wb = wb + mul_mv(iB, ang);
    }
    }  // revolute
    {
      V3 ra = rotate(sa.dq, j.frame_a.p), rb = rotate(sb.dq, j.frame_b.p);
      V3 cdot = (vb + cross(wb, rb)) - va - cross(wa, ra);
      V3 bias = v3(0, 0, 0);
      real ms = 1.0f, is = 0.0f;
      if (use_bias) {
        V3 dca = sa.dp, dcb = sb.dp;
        V3 sep = ((dcb - dca) + (rb - ra)) + j.delta_center;
        bias = j.constraint_softness.bias_rate * sep;
        ms = j.constraint_softness.mass_scale;
        is = j.constraint_softness.impulse_scale;
      }
      V3 b = solve_point_constraint(mA, mB, j.inv_ia, j.inv_ib, ra, rb, cdot + bias);
      V3 imp = (-ms) * b - is * j.linear_impulse;
      j.linear_impulse = j.linear_impulse + imp;
      va = va - mA * imp;
      wa = wa - mul_mv(iA, cross(ra, imp));
      vb = vb + mB * imp;
      wb = wb + mul_mv(iB, cross(rb, imp));
    }
    if (sa.flags & 0x1000u) { sa.v = va; sa.w = wa; }
    if (sb.flags & 0x1000u) { sb.v = vb; sb.w = wb; }
    if (j.index_a >= 0 && (sa.flags & 0x1000u)) states[j.index_a] = sa;
    if (j.index_b >= 0 && (sb.flags & 0x1000u)) states[j.index_b] = sb;
  }
}

}  // namespace nso
