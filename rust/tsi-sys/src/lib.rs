//! Raw bindings to include/tsi.h for the reference's Rust host.
//!
//! `GPUInstruction` here is layout-identical to `ir::GPUInstruction`
//! (src/ir.rs:88-97) and `Uniforms` to `uniforms::Uniforms`
//! (src/uniforms.rs:6-17), so the host passes its existing values through
//! unchanged.  Not compiled in this repository's CI
//! (no Rust toolchain on the build machines).
#![allow(non_camel_case_types)]
use std::os::raw::{c_char, c_float, c_int, c_void};

pub type tsi_status = c_int;
pub const TSI_OK: tsi_status = 0;

#[repr(C)]
#[derive(Debug, Copy, Clone, bytemuck::Pod, bytemuck::Zeroable)]
pub struct GPUInstruction {
    pub index_: u32,
    pub opcode_uses: u32,
    pub larg_rarg: u32,
    pub literal: f32,
    pub val: [f32; 2],
    pub sens: [f32; 2],
}

#[repr(C)]
#[derive(Debug, Copy, Clone)]
pub struct tsi_params {
    pub localsubdiv: i32,
    pub delta: f32,
    pub pointsample: i32,
    pub fastenabled: i32,
    pub lipschitz_corrected: i32,
    pub swept_volume: i32,
    pub fast_normals: i32,
    pub normal_viz: i32,
    pub rounding_mode: i32,
    pub fast_multiplier: f32,
    pub scene_id: i32,
    pub octree_darken_factor: f32,
    pub root_lo: [f32; 3],
    pub root_hi: [f32; 3],
    pub pruning: i32,
    pub swept_dt: f32,
}

#[repr(C)]
#[derive(Debug, Copy, Clone, bytemuck::Pod, bytemuck::Zeroable)]
pub struct Uniforms {
    pub view_matrix: [[f32; 4]; 4],
    pub resolution: [u32; 2],
    pub time: f32,
    pub lasttime: f32,
    pub rendermode: f32,
    pub _padding: [f32; 3],
}

#[repr(C)]
#[derive(Debug, Copy, Clone, Default)]
pub struct tsi_stats {
    pub parents_expanded: u64,
    pub cells_evaluated: u64,
    pub cells_reverse: u64,
    pub cells_skipped: u64,
    pub cells_ambiguous: u64,
    pub cells_empty: u64,
    pub cells_full: u64,
    pub cells_enqueued: u64,
    pub cells_reused: u64,
    pub instr_forward: u64,
    pub instr_reverse: u64,
    pub instr_full_equiv: u64,
    pub fp32_ops: u64,
    pub bricks_allocated: u64,
    pub bricks_freed: u64,
    pub voxels_live: u64,
    pub items_high_water: u64,
    pub tape_words: u64,
    pub prune_fallbacks: u64,
    pub levels: u32,
    pub error_flags: u32,
    pub device_ms: f32,
    pub reserved: f32,
}

#[repr(C)]
pub struct tsi_image {
    pub width: u32,
    pub height: u32,
    pub rgba: *mut c_float,
    pub depth: *mut c_float,
    pub normal: *mut c_float,
}

#[repr(C)]
pub struct tsi_device_opts {
    pub device: i32,
    pub work_item_capacity: u64,
    pub tape_arena_words: u64,
    pub log_arena_bytes: u64,
    pub watchdog_iters: u32,
    pub max_scenes_per_launch: u32,
}

pub enum tsi_ctx {}
pub enum tsi_tape {}
pub enum tsi_scene {}

extern "C" {
    pub fn tsi_version() -> u32;
    pub fn tsi_status_string(s: tsi_status) -> *const c_char;
    pub fn tsi_last_error() -> *const c_char;
    pub fn tsi_default_params(p: *mut tsi_params);
    pub fn tsi_create(opts: *const tsi_device_opts, out: *mut *mut tsi_ctx) -> tsi_status;
    pub fn tsi_destroy(ctx: *mut tsi_ctx);
    pub fn tsi_tape_upload(ctx: *mut tsi_ctx, instr: *const GPUInstruction, n: u32, out: *mut *mut tsi_tape) -> tsi_status;
    pub fn tsi_tape_from_llvm_ir(ctx: *mut tsi_ctx, text: *const c_char, len: usize, out: *mut *mut tsi_tape) -> tsi_status;
    pub fn tsi_tape_destroy(t: *mut tsi_tape);
    pub fn tsi_scene_create(ctx: *mut tsi_ctx, tape: *const tsi_tape, p: *const tsi_params, voxel_capacity: u64,
                            out: *mut *mut tsi_scene) -> tsi_status;
    pub fn tsi_scene_destroy(s: *mut tsi_scene);
    pub fn tsi_scene_reset(s: *mut tsi_scene) -> tsi_status;
    pub fn tsi_scene_invert(s: *mut tsi_scene, time: f32, t0_or_nan: f32, stats: *mut tsi_stats) -> tsi_status;
    pub fn tsi_scene_trace(s: *mut tsi_scene, u: *const Uniforms, out: *mut tsi_image, stats: *mut tsi_stats) -> tsi_status;
}

/// Convenience used by `State::compute`: one frame, returns device ms.
pub unsafe fn invert_frame(scene: *mut tsi_scene, time: f32) -> Result<f32, tsi_status> {
    let mut st = tsi_stats::default();
    let s = tsi_scene_invert(scene, time, f32::NAN, &mut st);
    if s == TSI_OK { Ok(st.device_ms) } else { Err(s) }
}

#[allow(dead_code)]
fn _assert_layouts() {
    let _: [u8; 32] = [0; std::mem::size_of::<GPUInstruction>()];
    let _: [u8; 96] = [0; std::mem::size_of::<Uniforms>()];
    let _ = std::ptr::null::<c_void>();
}
