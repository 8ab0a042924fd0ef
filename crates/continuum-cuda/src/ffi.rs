//! The C ABI of libcontinuum_cuda.so, declared one for one from
//! include/continuum_cuda.h (the header documents each call).

#![allow(non_camel_case_types)]

use std::os::raw::{c_char, c_int, c_void};

pub const CC_OK: c_int = 0;
pub const CC_ERR_INVALID: c_int = 1;
pub const CC_ERR_CUDA: c_int = 2;
pub const CC_ERR_OOM: c_int = 3;
pub const CC_ERR_NO_DEVICE: c_int = 4;
pub const CC_ERR_STACK: c_int = 5;
pub const CC_ERR_TIMEOUT: c_int = 6;
pub const CC_ERR_BUSY: c_int = 7;

pub const CC_NONE: u32 = 0xffff_ffff;

/// cc_options.flags
pub const CC_DEVICE_POINTERS: u32 = 1;
pub const CC_NO_REDO: u32 = 2;
pub const CC_KEEP_ORDER: u32 = 4;
pub const CC_NO_OBJECT_PREFILTER: u32 = 8;
pub const CC_BACK_FACING: u32 = 16;
/// cc_batch_options.flags
pub const CC_BATCH_GRAPH: u32 = 8;
/// cc_sky_visibility flags
pub const CC_SKY_COMBINE_MAX: u32 = 1;
pub const CC_SKY_NO_HORIZON_CULL: u32 = 2;
pub const CC_SKY_OBJECT_FRAME: u32 = 4;

/// Status bits of a cone (the fourth word of cc_outputs.work).
pub const CC_CONE_CAPPED: u32 = 1;
pub const CC_CONE_STACK: u32 = 2;
pub const CC_CONE_DIVERGED: u32 = 4;
pub const CC_CONE_REWALKED: u32 = 8;
pub const CC_CONE_FULL_STOP: u32 = 16;
pub const CC_CONE_ACC_WIDE: u32 = 32;

pub const CC_STATIC_MAX_CONES: u32 = 131_072;

#[repr(C)]
pub struct cc_context {
    _p: [u8; 0],
}
#[repr(C)]
pub struct cc_scene {
    _p: [u8; 0],
}
#[repr(C)]
pub struct cc_batch {
    _p: [u8; 0],
}
#[repr(C)]
pub struct cc_server {
    _p: [u8; 0],
}
#[repr(C)]
pub struct cc_cache {
    _p: [u8; 0],
}
#[repr(C)]
pub struct cc_planner {
    _p: [u8; 0],
}

/// The reference's `Flat` + `mesh_hierarchy` arrays (hierarchy.rs:11-66).
#[repr(C)]
pub struct cc_flat_scene {
    pub tris: *const f32,
    pub ntris: u32,
    pub ranges: *const u32,
    pub nmeshes: u32,
    pub blas: *const c_void,
    pub nblas: u32,
    pub blas_items: *const u32,
    pub nblas_items: u32,
    pub nodes: *const c_void,
    pub nnodes: u32,
    pub items: *const u32,
    pub nitems: u32,
    pub xforms: *const f32,
    pub nxforms: u32,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct cc_instance {
    pub geometry: u32,
    pub rotation: [f32; 9],
    pub scale: f32,
    pub translation: [f32; 3],
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct cc_options {
    pub hierarchy: u32,
    pub wide_extent: f32,
    pub light_cone_cap: u32,
    pub wide_cone_cap: u32,
    pub points_per_warp: u32,
    pub flags: u32,
    pub prefilter: f32,
}

#[repr(C)]
pub struct cc_outputs {
    pub full: *mut u32,
    pub any: *mut u32,
    pub partial: *mut f32,
    pub irradiance: *mut f32,
    pub fraction: *mut f32,
    pub work: *mut u32,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct cc_batch_options {
    pub points_per_warp: u32,
    pub blocks_per_sm: u32,
    pub flags: u32,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct cc_server_options {
    pub hbm_budget: u64,
    pub max_inflight: u32,
    pub max_queue: u32,
    pub max_launch_cones: u64,
    pub points_per_warp: u32,
    pub blocks_per_sm: u32,
    pub deadline_ns_per_cone: u32,
}

#[repr(C)]
pub struct cc_request {
    pub scene: u32,
    pub receivers: *const f32,
    pub npoints: u64,
    pub lights: *const f32,
    pub nlights: u32,
    pub hierarchy: u32,
    pub cache_key: u64,
    pub full: *mut u32,
    pub any: *mut u32,
    pub irradiance: *mut f32,
    pub fraction: *mut f32,
    pub prefilter: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Default)]
pub struct cc_request_stats {
    pub queued_ms: f64,
    pub total_ms: f64,
    pub launch_requests: u32,
    pub cached_lights: u32,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct cc_cache_options {
    pub pages: u32,
    pub bake_budget: u32,
    pub frame_target_ms: f32,
    pub frame_budget_ms: f32,
    pub floor_overrun: f32,
    pub light_ratio: u32,
}

#[repr(C)]
pub struct cc_page_request {
    pub key: [u32; 3],
    pub priority: u32,
    pub inside: [u32; 2],
    pub texels: *const f32,
}

#[repr(C)]
#[derive(Clone, Copy, Default)]
pub struct cc_cache_frame_info {
    pub period_ms: f32,
    pub render_ms: f32,
    pub gpu_waited: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Default)]
pub struct cc_cache_stats {
    pub budget: f32,
    pub frame: u32,
    pub pages_planned: u32,
    pub jobs: u32,
    pub spent: u32,
    pub resident: u32,
    pub evicted: u32,
    pub last_bake_ms: f32,
}

unsafe extern "C" {
    pub fn cc_context_create(device: c_int, out: *mut *mut cc_context) -> c_int;
    pub fn cc_context_destroy(ctx: *mut cc_context) -> c_int;
    pub fn cc_context_set_split_chunk(ctx: *mut cc_context, cones: u64) -> c_int;
    pub fn cc_last_error() -> *const c_char;

    pub fn cc_scene_upload(ctx: *mut cc_context, flat: *const cc_flat_scene, out: *mut *mut cc_scene) -> c_int;
    pub fn cc_scene_build(ctx: *mut cc_context, tri9: *const f32, mesh_counts: *const u32, nmeshes: u32,
                          out: *mut *mut cc_scene) -> c_int;
    pub fn cc_scene_destroy(scene: *mut cc_scene) -> c_int;
    pub fn cc_scene_build_instanced(ctx: *mut cc_context, tri9: *const f32, geometry_counts: *const u32,
                                    ngeometries: u32, instances: *const cc_instance, ninstances: u32,
                                    movable: *const u32, nmovable: u32, out: *mut *mut cc_scene) -> c_int;
    pub fn cc_scene_move(scene: *mut cc_scene, placements: *const cc_instance, nplacements: u32,
                         boxes12: *mut f32) -> c_int;
    pub fn cc_scene_set_clear(scene: *mut cc_scene, clear: *const f32, nobjects: u32) -> c_int;
    pub fn cc_stale_cones(ctx: *mut cc_context, scene: *const cc_scene, receivers: *const f32, npoints: u64,
                          lights: *const f32, nlights: u32, boxes12: *const f32, nmovers: u32, stale: *mut u8,
                          count: *mut u64, stream: *mut c_void) -> c_int;
    pub fn cc_scene_transforms(scene: *const cc_scene, out16: *mut f32, max_transforms: u64) -> u64;
    pub fn cc_scene_sizes(scene: *const cc_scene, out6: *mut u64) -> c_int;
    pub fn cc_scene_arrays(scene: *const cc_scene, ranges: *mut u32, blas: *mut c_void, blas_items: *mut u32,
                           nodes: *mut c_void, items: *mut u32) -> c_int;
    pub fn cc_scene_device_bytes(scene: *const cc_scene) -> u64;
    pub fn cc_scene_primary_hits(scene: *const cc_scene, camera: *const f32, width: u32, height: u32,
                                 out8: *mut f32, hit: *mut u8) -> c_int;

    pub fn cc_options_default(opt: *mut cc_options);
    pub fn cc_visibility(ctx: *mut cc_context, scene: *const cc_scene, receivers: *const f32, npoints: u64,
                         lights: *const f32, nlights: u32, opt: *const cc_options, out: *const cc_outputs,
                         stream: *mut c_void) -> c_int;
    pub fn cc_scene_coverage(scene: *const cc_scene, blas27: *mut f32, max_blas: u64, obj27: *mut f32,
                             max_obj: u64) -> i64;
    pub fn cc_sky_visibility(ctx: *mut cc_context, scene: *const cc_scene, receivers: *const f32, npoints: u64,
                             opt: *const cc_options, sky_flags: u32, irradiance: *mut f32, faces: *const cc_outputs,
                             stream: *mut c_void) -> c_int;
    pub fn cc_visibility_update(ctx: *mut cc_context, scene: *const cc_scene, receivers: *const f32, npoints: u64,
                                lights: *const f32, nlights: u32, stale: *const u8, opt: *const cc_options,
                                out: *const cc_outputs, recomputed: *mut u64, stream: *mut c_void) -> c_int;
    pub fn cc_visibility_static(scene: *const cc_scene, receivers: *const f32, npoints: u64, lights: *const f32,
                                nlights: u32, opt: *const cc_options, out: *const cc_outputs,
                                stream: *mut c_void) -> c_int;

    pub fn cc_batch_options_default(opt: *mut cc_batch_options);
    pub fn cc_batch_create(ctx: *mut cc_context, out: *mut *mut cc_batch) -> c_int;
    pub fn cc_batch_destroy(batch: *mut cc_batch) -> c_int;
    pub fn cc_batch_clear(batch: *mut cc_batch) -> c_int;
    pub fn cc_batch_add(batch: *mut cc_batch, scene: *const cc_scene, receivers: *const f32, npoints: u64,
                        lights: *const f32, nlights: u32, opt: *const cc_options, out: *const cc_outputs,
                        job: *mut u32) -> c_int;
    pub fn cc_batch_add_update(batch: *mut cc_batch, scene: *const cc_scene, receivers: *const f32, npoints: u64,
                               lights: *const f32, nlights: u32, stale: *const u8, opt: *const cc_options,
                               out: *const cc_outputs, job: *mut u32) -> c_int;
    pub fn cc_batch_submit(batch: *mut cc_batch, opt: *const cc_batch_options, stream: *mut c_void) -> c_int;
    pub fn cc_batch_wait(batch: *mut cc_batch, timeout_ms: u32) -> c_int;
    pub fn cc_batch_tune(batch: *mut cc_batch, base: *const cc_batch_options, reps: u32,
                         best: *mut cc_batch_options, ms_out: *mut f32, max_candidates: u32) -> c_int;
    pub fn cc_batch_sizes(batch: *const cc_batch, out4: *mut u64) -> c_int;

    pub fn cc_server_options_default(opt: *mut cc_server_options);
    pub fn cc_server_create(ctx: *mut cc_context, opt: *const cc_server_options, out: *mut *mut cc_server) -> c_int;
    pub fn cc_server_destroy(server: *mut cc_server) -> c_int;
    pub fn cc_server_add_scene(server: *mut cc_server, scene: *const cc_scene, id: *mut u32) -> c_int;
    pub fn cc_server_submit(server: *mut cc_server, req: *const cc_request, ticket: *mut u64) -> c_int;
    pub fn cc_server_wait(server: *mut cc_server, ticket: u64, timeout_ms: u32, stats: *mut cc_request_stats)
                          -> c_int;
    pub fn cc_server_stats(server: *mut cc_server, out8: *mut u64) -> c_int;

    pub fn cc_context_kernel_times(ctx: *mut cc_context, out2: *mut f32, max_calls: c_int) -> c_int;
    pub fn cc_irradiance(ctx: *mut cc_context, receivers6: *const f32, npoints: u64, light9: *const f32,
                         one_sided: c_int, tri9: *const f32, mesh_counts: *const u32, nmeshes: u32, hierarchy: u32,
                         runs: u32, out: *mut f32, best_seconds: *mut f64) -> c_int;
    pub fn cc_coverage(ctx: *mut cc_context, receivers6: *const f32, npoints: u64, light9: *const f32,
                       one_sided: c_int, tri9: *const f32, mesh_counts: *const u32, nmeshes: u32, out64: *mut f32)
                       -> c_int;

    pub fn cc_cache_options_default(opt: *mut cc_cache_options);
    pub fn cc_cache_create(ctx: *mut cc_context, scene: *const cc_scene, lights: *const f32, nlights: u32,
                           opt: *const cc_cache_options, out: *mut *mut cc_cache) -> c_int;
    pub fn cc_cache_destroy(cache: *mut cc_cache) -> c_int;
    pub fn cc_cache_frame(cache: *mut cc_cache, requests: *const cc_page_request, nrequests: u32,
                          info: *const cc_cache_frame_info, stats: *mut cc_cache_stats) -> c_int;
    pub fn cc_cache_read(cache: *mut cc_cache, key: *const u32, out: *mut f32) -> c_int;
    pub fn cc_cache_pool(cache: *mut cc_cache, pool: *mut *mut f32, channels: *mut u32) -> c_int;
    pub fn cc_cache_jobs(cache: *mut cc_cache, jobs2: *mut u32, max_jobs: u64, page_slots: *mut u32,
                         max_pages: u32) -> i64;
    pub fn cc_planner_create(opt: *const cc_cache_options, nlights: u32, out: *mut *mut cc_planner) -> c_int;
    pub fn cc_planner_destroy(planner: *mut cc_planner) -> c_int;
    pub fn cc_planner_frame(planner: *mut cc_planner, requests: *const cc_page_request, nrequests: u32,
                            info: *const cc_cache_frame_info, bake_ms: f32, stats: *mut cc_cache_stats) -> c_int;
    pub fn cc_planner_jobs(planner: *mut cc_planner, jobs2: *mut u32, max_jobs: u64, page_slots: *mut u32,
                           max_pages: u32) -> i64;
    pub fn cc_planner_slot(planner: *mut cc_planner, key: *const u32) -> i64;
}
