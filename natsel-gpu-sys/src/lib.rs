//! FFI bindings to `libnatsel_gpu.so`, the B200 rigid-body step declared in
//! `include/natsel_gpu.h`, and the safe pieces a host engine uses around them: an owning
//! [`GpuWorld`] and the rollout [`Tape`] guard.
//!
//! The reference engine keeps its `World` (src/simulation/world_runtime.rs:942) and mirrors
//! every body, shape and joint into a `GpuWorld` in creation order, so ids agree; its
//! `World::step` (src/simulation/solver_integration.rs:807) then branches to
//! [`GpuWorld::step`] and reads the bodies back. Every call returns 0 or an `NS_ERR_*` status,
//! with a message from `ns_last_error`; nothing panics across the boundary.
#![allow(non_camel_case_types)]

use std::ffi::CStr;
use std::os::raw::{c_char, c_int, c_void};

pub const NS_OK: c_int = 0;
pub const NS_ERR_INVALID: c_int = 1;
pub const NS_ERR_CUDA: c_int = 2;
pub const NS_ERR_CAPACITY: c_int = 3;
pub const NS_ERR_TIMEOUT: c_int = 4;
pub const NS_ERR_NONFINITE: c_int = 5;
pub const NS_ERR_UNSUPPORTED: c_int = 6;

pub const NS_STATIC_BODY: c_int = 0;
pub const NS_KINEMATIC_BODY: c_int = 1;
pub const NS_DYNAMIC_BODY: c_int = 2;

#[repr(C)]
pub struct ns_world {
    _private: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ns_world_def {
    pub gravity: [f32; 3],
    pub enable_sleep: c_int,
    pub enable_continuous: c_int,
    pub enable_warm_starting: c_int,
    pub contact_hertz: f32,
    pub contact_damping_ratio: f32,
    pub contact_speed: f32,
    pub max_linear_speed: f32,
    pub restitution_threshold: f32,
    pub restitution_iterations: c_int,
    pub joint_hertz: f32,
    pub joint_damping_ratio: f32,
    pub contact_capacity: c_int,
    pub solver_blocks: c_int,
    pub device: c_int,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ns_body_def {
    pub type_: c_int,
    pub position: [f64; 3],
    pub rotation: [f32; 4],
    pub linear_velocity: [f32; 3],
    pub angular_velocity: [f32; 3],
    pub linear_damping: f32,
    pub angular_damping: f32,
    pub gravity_scale: f32,
    pub enable_sleep: c_int,
    pub is_bullet: c_int,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ns_shape_def {
    pub density: f32,
    pub friction: f32,
    pub restitution: f32,
    pub rolling_resistance: f32,
    pub category_bits: u64,
    pub mask_bits: u64,
    pub group_index: c_int,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ns_revolute_joint_def {
    pub body_a: c_int,
    pub body_b: c_int,
    pub local_frame_a: [f32; 7],
    pub local_frame_b: [f32; 7],
    pub constraint_hertz: f32,
    pub constraint_damping_ratio: f32,
    pub collide_connected: c_int,
    pub target_angle: f32,
    pub enable_spring: c_int,
    pub hertz: f32,
    pub damping_ratio: f32,
    pub enable_limit: c_int,
    pub lower_angle: f32,
    pub upper_angle: f32,
    pub enable_motor: c_int,
    pub max_motor_torque: f32,
    pub motor_speed: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ns_spherical_joint_def {
    pub body_a: c_int,
    pub body_b: c_int,
    pub local_frame_a: [f32; 7],
    pub local_frame_b: [f32; 7],
    pub constraint_hertz: f32,
    pub constraint_damping_ratio: f32,
    pub collide_connected: c_int,
    pub enable_spring: c_int,
    pub hertz: f32,
    pub damping_ratio: f32,
    pub target_rotation: [f32; 4],
    pub enable_cone_limit: c_int,
    pub cone_angle: f32,
    pub enable_twist_limit: c_int,
    pub lower_twist_angle: f32,
    pub upper_twist_angle: f32,
    pub enable_motor: c_int,
    pub max_motor_torque: f32,
    pub motor_velocity: [f32; 3],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ns_pair_job {
    pub type_a: i32,
    pub type_b: i32,
    pub geom_a: [f32; 7],
    pub geom_b: [f32; 7],
    pub xf: [f32; 7],
    pub sat_separation: f32,
    pub sat_type: i32,
    pub sat_index_a: i32,
    pub sat_index_b: i32,
    pub sat_hit: i32,
    pub simplex_metric: f32,
    pub simplex_count: i32,
    pub simplex_ia: [i32; 4],
    pub simplex_ib: [i32; 4],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ns_pair_result {
    pub normal: [f32; 3],
    pub point_count: i32,
    pub points: [[f32; 4]; 4],
    pub feature_ids: [u32; 4],
}

extern "C" {
    pub fn ns_default_world_def(def: *mut ns_world_def);
    pub fn ns_world_create(def: *const ns_world_def) -> *mut ns_world;
    pub fn ns_world_destroy(world: *mut ns_world);
    pub fn ns_last_error(world: *const ns_world) -> *const c_char;

    pub fn ns_create_body(world: *mut ns_world, def: *const ns_body_def) -> c_int;
    pub fn ns_create_box_shape(world: *mut ns_world, body: c_int, def: *const ns_shape_def, hx: f32, hy: f32,
                               hz: f32) -> c_int;
    pub fn ns_create_sphere_shape(world: *mut ns_world, body: c_int, def: *const ns_shape_def, center: *const f32,
                                  radius: f32) -> c_int;
    pub fn ns_create_capsule_shape(world: *mut ns_world, body: c_int, def: *const ns_shape_def,
                                   center1: *const f32, center2: *const f32, radius: f32) -> c_int;
    pub fn ns_create_revolute_joint(world: *mut ns_world, body_a: c_int, body_b: c_int, frame_a: *const f32,
                                    frame_b: *const f32, enable_limit: c_int, lower_angle: f32, upper_angle: f32,
                                    enable_spring: c_int, hertz: f32, damping_ratio: f32, max_motor_torque: f32,
                                    collide_connected: c_int) -> c_int;
    pub fn ns_default_revolute_joint_def(def: *mut ns_revolute_joint_def);
    pub fn ns_create_revolute_joint_def(world: *mut ns_world, def: *const ns_revolute_joint_def) -> c_int;
    pub fn ns_default_spherical_joint_def(def: *mut ns_spherical_joint_def);
    pub fn ns_create_spherical_joint_def(world: *mut ns_world, def: *const ns_spherical_joint_def) -> c_int;

    pub fn ns_world_begin_subworld(world: *mut ns_world) -> c_int;
    pub fn ns_world_subworld_count(world: *const ns_world) -> c_int;
    pub fn ns_world_subworld_bodies(world: *const ns_world, first_body: *mut c_int) -> c_int;
    pub fn ns_world_subworld_hashes(world: *mut ns_world, out: *mut u64) -> c_int;

    pub fn ns_world_step(world: *mut ns_world, dt: f32, substeps: c_int) -> c_int;
    pub fn ns_world_apply_forces(world: *mut ns_world, force: *const f32, torque: *const f32) -> c_int;
    pub fn ns_world_synchronize(world: *mut ns_world) -> c_int;
    pub fn ns_world_get_bodies(world: *mut ns_world, pos: *mut f64, rot: *mut f32, lin: *mut f32,
                               ang: *mut f32) -> c_int;
    pub fn ns_world_body_count(world: *const ns_world) -> c_int;
    pub fn ns_world_state_hash(world: *mut ns_world, out_hash: *mut u64) -> c_int;
    pub fn ns_world_contact_capacity(world: *mut ns_world) -> c_int;
    pub fn ns_world_get_contacts(world: *mut ns_world, ints: *mut i32, features: *mut u32, floats: *mut f32,
                                 capacity: c_int) -> c_int;
    pub fn ns_world_counters(world: *mut ns_world, counters: *mut i32) -> c_int;
    pub fn ns_world_phase_times(world: *mut ns_world, ms5: *mut f32) -> c_int;
    pub fn ns_world_stream(world: *mut ns_world) -> *mut c_void;
    pub fn ns_world_solver_counts(world: *mut ns_world, counts16: *mut i64) -> c_int;

    pub fn ns_collide_pairs(jobs: *mut ns_pair_job, results: *mut ns_pair_result, count: c_int) -> c_int;
    pub fn ns_collide_pairs_noalloc(jobs: *mut ns_pair_job, results: *mut ns_pair_result, count: c_int) -> c_int;
    pub fn ns_selftest_barrier_timeout(device: c_int, timeout_ms: c_int) -> c_int;

    pub fn ns_world_autotune(w: *mut ns_world, dt: f32, substeps: c_int, steps: c_int, blocks_out: *mut c_int,
                             grid_out: *mut c_int, ms_out: *mut f32, max_candidates: c_int) -> c_int;
    pub fn ns_world_autotune_table(w: *const ns_world, dimension: *mut c_int, value_a: *mut c_int,
                                   value_b: *mut c_int, ms: *mut f32, max_rows: c_int) -> c_int;
    pub fn ns_world_launch_shapes(w: *const ns_world, out8: *mut c_int) -> c_int;
    pub fn ns_world_set_launch_shapes(w: *mut ns_world, in8: *const c_int) -> c_int;

    pub fn ns_world_tape_begin(w: *mut ns_world, checkpoint_substeps: c_int) -> c_int;
    pub fn ns_world_tape_end(w: *mut ns_world) -> c_int;
    pub fn ns_world_tape_free(w: *mut ns_world) -> c_int;
    pub fn ns_world_tape_info(w: *mut ns_world, out: *mut i64) -> c_int;
    pub fn ns_world_vjp(w: *mut ns_world, dpos: *const f32, drot: *const f32, dlin: *const f32, dang: *const f32,
                        dlin0: *mut f32, dang0: *mut f32, dmass: *mut f32, dfriction: *mut f32, dpos0: *mut f32,
                        drot0: *mut f32) -> c_int;
    pub fn ns_world_vjp_restitution(w: *const ns_world, drestitution: *mut f32) -> c_int;
    pub fn ns_world_vjp_f64(w: *mut ns_world, dpos: *const f32, drot: *const f32, dlin: *const f32,
                            dang: *const f32, dlin0: *mut f64, dang0: *mut f64, dmass: *mut f64,
                            dfriction: *mut f64, dpos0: *mut f64, drot0: *mut f64) -> c_int;
    pub fn ns_adjoint_selfcheck(which: c_int, seed: c_int, worst: *mut f64) -> c_int;
}

/// A failed call: its status and the library's message.
#[derive(Clone, Debug)]
pub struct NsError {
    pub code: c_int,
    pub message: String,
}

fn check(code: c_int, w: *const ns_world) -> Result<(), NsError> {
    if code == NS_OK {
        return Ok(());
    }
    let message = unsafe {
        let p = ns_last_error(w);
        if p.is_null() { String::new() } else { CStr::from_ptr(p).to_string_lossy().into_owned() }
    };
    Err(NsError { code, message })
}

/// An owning handle of one device world. Like the reference `World` it is `Send` but not
/// `Sync`: calls on one world are serialised by `&mut self`.
pub struct GpuWorld {
    ptr: *mut ns_world,
    pos: Vec<f64>,
    rot: Vec<f32>,
    lin: Vec<f32>,
    ang: Vec<f32>,
}

unsafe impl Send for GpuWorld {}

impl GpuWorld {
    /// The reference World::new defaults (world_runtime.rs:1243-1272) with `edit` applied.
    pub fn new(edit: impl FnOnce(&mut ns_world_def)) -> Result<Self, NsError> {
        let mut def = ns_world_def::default();
        unsafe { ns_default_world_def(&mut def) };
        edit(&mut def);
        let ptr = unsafe { ns_world_create(&def) };
        if ptr.is_null() {
            check(NS_ERR_INVALID, std::ptr::null())?;
        }
        Ok(GpuWorld { ptr, pos: Vec::new(), rot: Vec::new(), lin: Vec::new(), ang: Vec::new() })
    }

    pub fn raw(&mut self) -> *mut ns_world {
        self.ptr
    }

    fn id(&self, id: c_int) -> Result<i32, NsError> {
        if id < 0 { Err(check(NS_ERR_INVALID, self.ptr).unwrap_err()) } else { Ok(id) }
    }

    pub fn create_body(&mut self, def: &ns_body_def) -> Result<i32, NsError> {
        self.id(unsafe { ns_create_body(self.ptr, def) })
    }

    pub fn create_box(&mut self, body: i32, def: &ns_shape_def, half: [f32; 3]) -> Result<i32, NsError> {
        self.id(unsafe { ns_create_box_shape(self.ptr, body, def, half[0], half[1], half[2]) })
    }

    pub fn create_sphere(&mut self, body: i32, def: &ns_shape_def, center: [f32; 3], radius: f32) -> Result<i32, NsError> {
        self.id(unsafe { ns_create_sphere_shape(self.ptr, body, def, center.as_ptr(), radius) })
    }

    pub fn create_capsule(&mut self, body: i32, def: &ns_shape_def, c1: [f32; 3], c2: [f32; 3],
                          radius: f32) -> Result<i32, NsError> {
        self.id(unsafe { ns_create_capsule_shape(self.ptr, body, def, c1.as_ptr(), c2.as_ptr(), radius) })
    }

    pub fn create_revolute(&mut self, def: &ns_revolute_joint_def) -> Result<i32, NsError> {
        self.id(unsafe { ns_create_revolute_joint_def(self.ptr, def) })
    }

    pub fn create_spherical(&mut self, def: &ns_spherical_joint_def) -> Result<i32, NsError> {
        self.id(unsafe { ns_create_spherical_joint_def(self.ptr, def) })
    }

    /// The per-step external forces and torques (3 floats per body, body id order).
    pub fn apply_forces(&mut self, force: Option<&[f32]>, torque: Option<&[f32]>) -> Result<(), NsError> {
        let f = force.map_or(std::ptr::null(), |v| v.as_ptr());
        let t = torque.map_or(std::ptr::null(), |v| v.as_ptr());
        check(unsafe { ns_world_apply_forces(self.ptr, f, t) }, self.ptr)
    }

    /// World::step (solver_integration.rs:807) on the device; asynchronous until a readback.
    pub fn step(&mut self, dt: f32, substeps: i32) -> Result<(), NsError> {
        check(unsafe { ns_world_step(self.ptr, dt, substeps) }, self.ptr)
    }

    /// Positions (f64), rotations (x, y, z, s), linear and angular velocities of every body in
    /// id order, read back after the queued steps (device errors of those steps surface here).
    pub fn bodies(&mut self) -> Result<(&[f64], &[f32], &[f32], &[f32]), NsError> {
        let n = unsafe { ns_world_body_count(self.ptr) }.max(0) as usize;
        self.pos.resize(3 * n, 0.0);
        self.rot.resize(4 * n, 0.0);
        self.lin.resize(3 * n, 0.0);
        self.ang.resize(3 * n, 0.0);
        check(unsafe {
            ns_world_get_bodies(self.ptr, self.pos.as_mut_ptr(), self.rot.as_mut_ptr(), self.lin.as_mut_ptr(),
                                self.ang.as_mut_ptr())
        }, self.ptr)?;
        Ok((&self.pos, &self.rot, &self.lin, &self.ang))
    }

    /// World::world_state_hash (body_queries.rs:432), bit-identical to the reference's.
    pub fn state_hash(&mut self) -> Result<u64, NsError> {
        let mut h = 0u64;
        check(unsafe { ns_world_state_hash(self.ptr, &mut h) }, self.ptr)?;
        Ok(h)
    }

    /// Times the launch-shape candidates from a copy of the world and keeps the fastest (the
    /// device's counterpart of WorldDef::worker_count, world_def.rs:94). The world is unchanged.
    pub fn autotune(&mut self, dt: f32, substeps: i32, steps: i32) -> Result<(), NsError> {
        let r = unsafe {
            ns_world_autotune(self.ptr, dt, substeps, steps, std::ptr::null_mut(), std::ptr::null_mut(),
                              std::ptr::null_mut(), 0)
        };
        if r < 0 { check(-r, self.ptr) } else { Ok(()) }
    }
}

impl Drop for GpuWorld {
    fn drop(&mut self) {
        unsafe { ns_world_destroy(self.ptr) };
    }
}

/// Gradients at the start of a recorded rollout, 3 (or 1) values per body in id order.
pub struct Grads {
    pub lin0: Vec<f32>,
    pub ang0: Vec<f32>,
    pub mass: Vec<f32>,
    pub friction: Vec<f32>,
    pub restitution: Vec<f32>,
}

impl Grads {
    pub fn new(bodies: usize) -> Self {
        Grads { lin0: vec![0.0; 3 * bodies], ang0: vec![0.0; 3 * bodies], mass: vec![0.0; bodies],
                friction: vec![0.0; bodies], restitution: vec![0.0; bodies] }
    }
}

/// The rollout tape: records the steps taken through it (checkpoints every
/// `checkpoint_substeps` substeps) and pulls cotangents of the final state back to the
/// initial velocities, masses, frictions and restitutions. Dropping it releases the tape.
pub struct Tape<'a> {
    gpu: &'a mut GpuWorld,
}

impl<'a> Tape<'a> {
    pub fn begin(gpu: &'a mut GpuWorld, checkpoint_substeps: i32) -> Result<Self, NsError> {
        check(unsafe { ns_world_tape_begin(gpu.ptr, checkpoint_substeps) }, gpu.ptr)?;
        Ok(Tape { gpu })
    }

    pub fn step(&mut self, dt: f32, substeps: i32) -> Result<(), NsError> {
        self.gpu.step(dt, substeps)
    }

    /// Cotangents of the final positions (3 per body, body id order) to gradients at the start.
    pub fn vjp(&mut self, dpos: &[f32], grads: &mut Grads) -> Result<(), NsError> {
        check(unsafe {
            ns_world_vjp(self.gpu.ptr, dpos.as_ptr(), std::ptr::null(), std::ptr::null(), std::ptr::null(),
                         grads.lin0.as_mut_ptr(), grads.ang0.as_mut_ptr(), grads.mass.as_mut_ptr(),
                         grads.friction.as_mut_ptr(), std::ptr::null_mut(), std::ptr::null_mut())
        }, self.gpu.ptr)?;
        check(unsafe { ns_world_vjp_restitution(self.gpu.ptr, grads.restitution.as_mut_ptr()) }, self.gpu.ptr)
    }
}

impl Drop for Tape<'_> {
    fn drop(&mut self) {
        unsafe { ns_world_tape_free(self.gpu.ptr) };
    }
}
