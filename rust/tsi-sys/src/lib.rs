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
    pub cinematic: i32,
    pub samples: i32,
    pub see_background: i32,
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
    pub fp32_ops_full_fwd: u64,
    pub fp32_ops_full_rev: u64,
    pub cells_unpruned_regs: u64,
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
    pub wide_smem_bytes: u32,
    pub hbm_budget_bytes: u64,
}

#[repr(C)]
#[derive(Debug, Copy, Clone, Default)]
pub struct tsi_tape_info {
    pub instruction_count: u32,
    pub registers: u32,
    pub minmax_count: u32,
    pub reserved: u32,
}

#[repr(C)]
pub struct tsi_image_device {
    pub width: u32,
    pub height: u32,
    pub rgba: *const c_float,
    pub depth: *const c_float,
    pub normal: *const c_float,
}

#[repr(C)]
#[derive(Debug, Copy, Clone, Default)]
pub struct tsi_cell {
    pub level: u32,
    pub ix: u32,
    pub iy: u32,
    pub iz: u32,
    pub f: f32,
    pub t: f32,
    pub time_err: f32,
    pub fast: f32,
    pub dx: f32,
    pub dy: f32,
    pub dz: f32,
    pub has_children: u32,
    pub x: [f32; 2],
    pub y: [f32; 2],
    pub z: [f32; 2],
}

#[repr(C)]
#[derive(Debug, Copy, Clone, Default)]
pub struct tsi_leaf {
    pub level: u32,
    pub ix: u32,
    pub iy: u32,
    pub iz: u32,
}

pub const TSI_AUTOTUNE_MAX: usize = 16;
#[repr(C)]
#[derive(Debug, Copy, Clone, Default)]
pub struct tsi_autotune_result {
    pub wide_threshold: u32,
    pub candidates: u32,
    pub threshold: [u32; TSI_AUTOTUNE_MAX],
    pub ms: [f32; TSI_AUTOTUNE_MAX],
    pub deep_level: u32,
    pub deep_threshold: u32,
    pub narrow_parents: u32,
    pub wide_prune_level: u32,
}

/// Caller-owned device buffers of a composited frame (one animation split at the root).
#[repr(C)]
pub struct tsi_frame_device {
    pub width: u32,
    pub height: u32,
    pub rgba: *mut c_float,
    pub depth: *mut c_float,
    pub normal: *mut c_float,
    pub key: *mut u64,
}
pub const TSI_COMPOSITE_MAX: usize = 64;

#[repr(C)]
pub struct tsi_request {
    pub scene: *mut tsi_scene,
    pub time: f32,
    pub t0_or_nan: f32,
    pub uniforms: *const Uniforms,
    pub out: *mut tsi_image,
    pub stats: *mut tsi_stats,
}

#[repr(C)]
#[derive(Debug, Copy, Clone, Default)]
pub struct tsi_server_opts {
    pub max_batch: u32,
    pub flags: u32,
    pub max_queue: u32,
    pub reserved: u32,
}

#[repr(C)]
#[derive(Debug, Copy, Clone, Default)]
pub struct tsi_server_stats {
    pub completed: u64,
    pub batches: u64,
    pub mean_batch: f32,
    pub p50_ms: f32,
    pub p99_ms: f32,
    pub max_ms: f32,
    pub queued: u32,
}

pub const TSI_SERVER_STATIC_BATCHES: u32 = 1;

pub enum tsi_ctx {}
pub enum tsi_tape {}
pub enum tsi_scene {}
pub enum tsi_batch_graph {}
pub enum tsi_server {}

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
    pub fn tsi_synchronize(ctx: *mut tsi_ctx) -> tsi_status;
    pub fn tsi_ir_lower(text: *const c_char, len: usize, time: f32, out: *mut GPUInstruction, cap: u32, n: *mut u32)
                        -> tsi_status;
    pub fn tsi_tape_info_get(t: *const tsi_tape, info: *mut tsi_tape_info) -> tsi_status;
    pub fn tsi_tape_eval_boxes(ctx: *mut tsi_ctx, t: *const tsi_tape, n: u32, boxes: *const f32, rounding_mode: i32,
                               reverse: i32, out: *mut f32) -> tsi_status;
    pub fn tsi_scene_image_device(s: *mut tsi_scene, out: *mut tsi_image_device) -> tsi_status;
    pub fn tsi_scene_image_copy(s: *mut tsi_scene, out: *mut tsi_image) -> tsi_status;
    pub fn tsi_params_subtree(full: *const tsi_params, level: u32, index: u32, out: *mut tsi_params) -> tsi_status;
    pub fn tsi_frames_composite(ctx: *mut tsi_ctx, scenes: *const *mut tsi_scene, ids: *const u32, n: u32,
                                out: *mut tsi_frame_device) -> tsi_status;
    pub fn tsi_frame_keep_nearest(ctx: *mut tsi_ctx, global_key: *const u64, frame: *mut tsi_frame_device)
                                  -> tsi_status;
    pub fn tsi_scene_invert_async(s: *mut tsi_scene, time: f32, t0_or_nan: f32) -> tsi_status;
    pub fn tsi_scene_invert_wait(s: *mut tsi_scene, stats: *mut tsi_stats) -> tsi_status;
    pub fn tsi_scene_trace_async(s: *mut tsi_scene, u: *const Uniforms, out: *mut tsi_image) -> tsi_status;
    pub fn tsi_scene_trace_wait(s: *mut tsi_scene) -> tsi_status;
    pub fn tsi_tape_wide_threshold(t: *const tsi_tape) -> u32;
    pub fn tsi_tape_set_wide_threshold(t: *mut tsi_tape, min_len: u32) -> tsi_status;
    pub fn tsi_tape_set_wide_threshold_deep(t: *mut tsi_tape, level: u32, min_len: u32) -> tsi_status;
    pub fn tsi_tape_wide_threshold_deep(t: *const tsi_tape, level: *mut u32, min_len: *mut u32) -> tsi_status;
    pub fn tsi_tape_set_narrow_parents(t: *mut tsi_tape, parents: u32) -> tsi_status;
    pub fn tsi_tape_narrow_parents(t: *const tsi_tape) -> u32;
    pub fn tsi_tape_set_wide_prune_level(t: *mut tsi_tape, level: u32) -> tsi_status;
    pub fn tsi_tape_wide_prune_level(t: *const tsi_tape) -> u32;
    pub fn tsi_scene_autotune(s: *mut tsi_scene, times: *const f32, ntimes: u32, reps: u32,
                              out: *mut tsi_autotune_result) -> tsi_status;
    pub fn tsi_scene_readback_cells(s: *mut tsi_scene, out: *mut tsi_cell, cap: u64, n: *mut u64) -> tsi_status;
    pub fn tsi_scene_readback_leaves(s: *mut tsi_scene, out: *mut tsi_leaf, cap: u64, n: *mut u64) -> tsi_status;
    pub fn tsi_scene_snapshot_size(s: *mut tsi_scene, bytes: *mut u64) -> tsi_status;
    pub fn tsi_scene_snapshot(s: *mut tsi_scene, host: *mut c_void, cap: u64, bytes: *mut u64) -> tsi_status;
    pub fn tsi_scene_restore(s: *mut tsi_scene, host: *const c_void, bytes: u64) -> tsi_status;
    pub fn tsi_scene_get_params(s: *const tsi_scene, out: *mut tsi_params) -> tsi_status;
    pub fn tsi_scene_device_bytes(s: *const tsi_scene) -> u64;
    pub fn tsi_scenes_device_bytes(ctx: *const tsi_ctx) -> u64;
    pub fn tsi_batch_run(ctx: *mut tsi_ctx, reqs: *mut tsi_request, n: u32) -> tsi_status;
    pub fn tsi_batch_autotune(ctx: *mut tsi_ctx, reqs: *const tsi_request, n: u32, frames: u32,
                              out: *mut tsi_autotune_result) -> tsi_status;
    pub fn tsi_batch_graph_create(ctx: *mut tsi_ctx, reqs: *mut tsi_request, n: u32, out: *mut *mut tsi_batch_graph)
                                  -> tsi_status;
    pub fn tsi_batch_graph_launch(g: *mut tsi_batch_graph) -> tsi_status;
    pub fn tsi_batch_graph_wait(g: *mut tsi_batch_graph, stats: *mut tsi_stats) -> tsi_status;
    pub fn tsi_batch_graph_destroy(g: *mut tsi_batch_graph);
    pub fn tsi_server_create(ctx: *mut tsi_ctx, opts: *const tsi_server_opts, out: *mut *mut tsi_server) -> tsi_status;
    pub fn tsi_server_submit(s: *mut tsi_server, req: *const tsi_request, ticket: *mut u64) -> tsi_status;
    pub fn tsi_server_poll(s: *mut tsi_server, ticket: u64, wait_ms: u32, latency_ms: *mut f32) -> tsi_status;
    pub fn tsi_server_stats_get(s: *mut tsi_server, out: *mut tsi_server_stats) -> tsi_status;
    pub fn tsi_server_destroy(s: *mut tsi_server);
    pub fn tsi_tape_eval_boxes_static(t: *const tsi_tape, n: u32, boxes_dev: *const f32, rounding_mode: i32,
                                      reverse: i32, out_dev: *mut f32, stream: *mut c_void) -> tsi_status;
    pub fn tsi_static_scratch_bytes() -> u64;
    pub fn tsi_rgba8_from_frame(rgba: *const f32, n_pixels: u64, out: *mut u8);
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
