//! Continuum's mask-cone visibility on a B200, behind the calls that
//! `continuum_gpu::MaskConeKernel` serves with wgpu compute
//! (crates/continuum-gpu/src/lib.rs:1706-1730 and :3289-3298). Callers switch
//! by constructing a `CudaConeKernel` instead; the arguments and results are
//! the reference's. Errors are returned where the reference panics
//! (`expect("GPU poll failed")`, lib.rs:3509).

pub mod ffi;

use std::ffi::CStr;
use std::time::Duration;

use continuum::glam::Vec3;
use continuum_gpu::{Hierarchy, RectLight};

type Tri = [Vec3; 3];

/// A failed call: the library's status code and message.
#[derive(Debug, Clone)]
pub struct Error {
    pub code: i32,
    pub message: String,
}

impl std::fmt::Display for Error {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        write!(f, "continuum_cuda error {}: {}", self.code, self.message)
    }
}

impl std::error::Error for Error {}

fn check(code: i32) -> Result<(), Error> {
    if code == ffi::CC_OK {
        return Ok(());
    }
    let message = unsafe { CStr::from_ptr(ffi::cc_last_error()) }.to_string_lossy().into_owned();
    Err(Error { code, message })
}

fn receivers6(receivers: &[(Vec3, Vec3)]) -> Vec<f32> {
    receivers.iter().flat_map(|(p, n)| [p.x, p.y, p.z, n.x, n.y, n.z]).collect()
}

fn meshes9(meshes: &[Vec<Tri>]) -> (Vec<f32>, Vec<u32>) {
    let tris = meshes.iter().flatten().flat_map(|t| t.iter().flat_map(|v| [v.x, v.y, v.z])).collect();
    let counts = meshes.iter().map(|m| m.len() as u32).collect();
    (tris, counts)
}

fn light9(light: &RectLight) -> [f32; 9] {
    let (c, u, v) = (light.corner, light.edge_u, light.edge_v);
    [c.x, c.y, c.z, u.x, u.y, u.z, v.x, v.y, v.z]
}

/// The CUDA counterpart of `MaskConeKernel`. One context per device; like
/// the reference's kernel it is used from one thread at a time (`Send`, not
/// `Sync`) and serves one call at a time.
pub struct CudaConeKernel {
    ctx: *mut ffi::cc_context,
}

unsafe impl Send for CudaConeKernel {}

impl CudaConeKernel {
    /// `None` without a CUDA device, as `MaskConeKernel::new` without an adapter.
    pub fn new() -> Option<Self> {
        Self::on_device(0)
    }

    pub fn on_device(device: i32) -> Option<Self> {
        let mut ctx = std::ptr::null_mut();
        (unsafe { ffi::cc_context_create(device, &mut ctx) } == ffi::CC_OK).then_some(Self { ctx })
    }

    /// `MaskConeKernel::irradiance_with`: irradiance per unit radiance at each
    /// receiver, and the fastest of `runs` kernel executions.
    pub fn irradiance_with(&self, receivers: &[(Vec3, Vec3)], light: RectLight, meshes: &[Vec<Tri>],
                           hierarchy: impl Into<Hierarchy>, runs: usize) -> Result<(Vec<f32>, Duration), Error> {
        let rec = receivers6(receivers);
        let (tris, counts) = meshes9(meshes);
        let l9 = light9(&light);
        let mut out = vec![0.0f32; receivers.len()];
        let mut best = 0.0f64;
        check(unsafe {
            ffi::cc_irradiance(self.ctx, rec.as_ptr(), receivers.len() as u64, l9.as_ptr(), light.one_sided as i32,
                               tris.as_ptr(), counts.as_ptr(), counts.len() as u32, hierarchy.into() as u32,
                               runs.max(1) as u32, out.as_mut_ptr(), &mut best)
        })?;
        Ok((out, Duration::from_secs_f64(best)))
    }

    /// `MaskConeKernel::irradiance`: every triangle tested.
    pub fn irradiance(&self, receivers: &[(Vec3, Vec3)], light: RectLight, meshes: &[Vec<Tri>], runs: usize)
                      -> Result<(Vec<f32>, Duration), Error> {
        self.irradiance_with(receivers, light, meshes, Hierarchy::None, runs)
    }

    /// `MaskConeKernel::coverage`: the 64 per-bin coverages of each receiver's cone.
    pub fn coverage(&self, receivers: &[(Vec3, Vec3)], light: RectLight, meshes: &[Vec<Tri>])
                    -> Result<Vec<[f32; 64]>, Error> {
        let rec = receivers6(receivers);
        let (tris, counts) = meshes9(meshes);
        let l9 = light9(&light);
        let mut out = vec![[0.0f32; 64]; receivers.len()];
        check(unsafe {
            ffi::cc_coverage(self.ctx, rec.as_ptr(), receivers.len() as u64, l9.as_ptr(), light.one_sided as i32,
                             tris.as_ptr(), counts.as_ptr(), counts.len() as u32, out.as_mut_ptr().cast())
        })?;
        Ok(out)
    }

    /// A scene kept on the device across calls (the reference rebuilds and
    /// uploads it on every `run`, lib.rs:3330-3494).
    pub fn scene(&self, meshes: &[Vec<Tri>]) -> Result<Scene<'_>, Error> {
        let (tris, counts) = meshes9(meshes);
        let mut scene = std::ptr::null_mut();
        check(unsafe { ffi::cc_scene_build(self.ctx, tris.as_ptr(), counts.as_ptr(), counts.len() as u32,
                                           &mut scene) })?;
        Ok(Scene { kernel: self, scene })
    }
}

impl Drop for CudaConeKernel {
    fn drop(&mut self) {
        unsafe {
            ffi::cc_context_destroy(self.ctx);
        }
    }
}

/// Per-cone results of `Scene::visibility`, light-major (cone = light * points + point).
pub struct Visibility {
    /// Bins wholly covered, bin b = bit b.
    pub full: Vec<u64>,
    /// Bins with any coverage.
    pub any: Vec<u64>,
    /// Irradiance per unit radiance (hit_irradiance_rect, mask_cones.wgsl:2125-2128).
    pub irradiance: Vec<f32>,
    /// The lighting cache's visible fraction (vc_bake, mask_cones.wgsl:3453-3510).
    pub fraction: Vec<f32>,
}

/// A resident scene of a `CudaConeKernel`.
pub struct Scene<'k> {
    kernel: &'k CudaConeKernel,
    scene: *mut ffi::cc_scene,
}

impl Scene<'_> {
    /// Every (light, point) cone. `receivers`: 8 floats each (`ReceiverGpu`,
    /// lib.rs:54-60); `lights`: 16 floats each (`LightGpu`, lib.rs:710-749).
    pub fn visibility(&self, receivers: &[[f32; 8]], lights: &[[f32; 16]], hierarchy: impl Into<Hierarchy>)
                      -> Result<Visibility, Error> {
        let cones = receivers.len() * lights.len();
        let mut v = Visibility { full: vec![0; cones], any: vec![0; cones], irradiance: vec![0.0; cones],
                                 fraction: vec![0.0; cones] };
        let mut opt = std::mem::MaybeUninit::<ffi::cc_options>::uninit();
        let mut opt = unsafe {
            ffi::cc_options_default(opt.as_mut_ptr());
            opt.assume_init()
        };
        opt.hierarchy = hierarchy.into() as u32;
        let out = ffi::cc_outputs {
            full: v.full.as_mut_ptr().cast(),
            any: v.any.as_mut_ptr().cast(),
            partial: std::ptr::null_mut(),
            irradiance: v.irradiance.as_mut_ptr(),
            fraction: v.fraction.as_mut_ptr(),
            work: std::ptr::null_mut(),
        };
        check(unsafe {
            ffi::cc_visibility(self.kernel.ctx, self.scene, receivers.as_ptr().cast(), receivers.len() as u64,
                               lights.as_ptr().cast(), lights.len() as u32, &opt, &out, std::ptr::null_mut())
        })?;
        Ok(v)
    }
}

impl Drop for Scene<'_> {
    fn drop(&mut self) {
        unsafe {
            ffi::cc_scene_destroy(self.scene);
        }
    }
}

/// Many visibility jobs in one persistent launch (cc_batch_*). Jobs take
/// device pointers that must stay valid while the batch is submitted.
pub struct Batch<'k> {
    _kernel: &'k CudaConeKernel,
    batch: *mut ffi::cc_batch,
}

impl<'k> Batch<'k> {
    pub fn new(kernel: &'k CudaConeKernel) -> Result<Self, Error> {
        let mut batch = std::ptr::null_mut();
        check(unsafe { ffi::cc_batch_create(kernel.ctx, &mut batch) })?;
        Ok(Self { _kernel: kernel, batch })
    }

    /// Appends a job (device pointers: receivers, lights, outputs).
    ///
    /// # Safety
    /// Every pointer must be a device allocation of the sizes the header
    /// states and stay valid while the batch is submitted.
    pub unsafe fn add(&mut self, scene: &Scene<'_>, receivers: *const f32, npoints: u64, lights: *const f32,
                      nlights: u32, out: &ffi::cc_outputs) -> Result<u32, Error> {
        let mut job = 0u32;
        check(unsafe {
            ffi::cc_batch_add(self.batch, scene.scene, receivers, npoints, lights, nlights, std::ptr::null(), out,
                              &mut job)
        })?;
        Ok(job)
    }

    /// Enqueues the batch on the context's stream (replayed from a captured
    /// CUDA graph with CC_BATCH_GRAPH).
    pub fn submit(&mut self, opt: &ffi::cc_batch_options) -> Result<(), Error> {
        check(unsafe { ffi::cc_batch_submit(self.batch, opt, std::ptr::null_mut()) })
    }

    /// Waits at most `timeout` for the last submission (CC_ERR_TIMEOUT if it has not finished).
    pub fn wait(&mut self, timeout: Duration) -> Result<(), Error> {
        check(unsafe { ffi::cc_batch_wait(self.batch, timeout.as_millis().min(u32::MAX as u128) as u32) })
    }
}

impl Drop for Batch<'_> {
    fn drop(&mut self) {
        unsafe {
            ffi::cc_batch_destroy(self.batch);
        }
    }
}
