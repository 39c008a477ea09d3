//! Raw bindings to `include/sr_cuda.h`, the C ABI of the B200 field update, and a thin safe `Step` over them.
//!
//! This is the crate `sr-engine` depends on to swap its wgpu step for the CUDA one: `Step::run`
//! (crates/sr-engine/src/step/mod.rs:703-718) becomes `sr_step`, `State::upload`/`readback`
//! (crates/sr-engine/src/state.rs:251-279) become `sr_upload`/`sr_readback`, and a non-zero status maps onto the
//! engine's existing `FftError`/`StateError`/exit-code paths. Every declaration below mirrors one of the header's, in
//! the header's order and with its field order; the `struct_size` field and `sr_abi_version()` catch a mismatch at run
//! time.
#![allow(non_camel_case_types, non_snake_case, clippy::missing_safety_doc)]

use std::ffi::CStr;
use std::os::raw::{c_char, c_void};

pub const SR_ABI_VERSION: u32 = 3;

pub type sr_status = i32;
pub const SR_OK: sr_status = 0;
pub const SR_E_INVALID: sr_status = 1;
pub const SR_E_NONFINITE: sr_status = 2;
pub const SR_E_TIMEOUT: sr_status = 3;
pub const SR_E_CUDA: sr_status = 4;
pub const SR_E_NOMEM: sr_status = 5;
pub const SR_E_UNSUPPORTED: sr_status = 6;

pub const SR_EDGE_BOUNCE: u32 = 0;
pub const SR_EDGE_LEAVE: u32 = 1;
pub const SR_LIMITER_MC: u32 = 0;
pub const SR_LIMITER_MINMOD: u32 = 1;
pub const SR_KERNEL_SELF_CELL: u32 = 0;
pub const SR_KERNEL_SOFTENED: u32 = 1;
pub const SR_PRECOND_MG: u32 = 0;
pub const SR_PRECOND_JACOBI: u32 = 1;
pub const SR_PRECOND_LEARNED: u32 = 2;

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct sr_config {
    pub struct_size: u32,
    pub width: u32,
    pub height: u32,
    pub channels: u32,
    pub edge: u32,
    pub limiter: u32,
    pub thermal_bracket: u32,
    pub gravity: u32,
    pub hydro: u32,
    pub heat: u32,
    pub kernel: u32,
    pub precond: u32,
    pub flux_limiter: u32,
    pub opacity_plane: u32,
    pub mg_pre: u32,
    pub mg_post: u32,
    pub max_passes: u32,
    pub max_rounds: u32,
    pub pin_temperature: u32,
    pub active_box: u32,
    pub reserved: [u32; 3],
    pub gamma: f64,
    pub mu: f64,
    pub t_floor: f64,
    pub sigma_vac: f64,
    pub sigma_floor: f64,
    pub cfl: f64,
    pub eta_g: f64,
    pub G: f64,
    pub softening: f64,
    pub a_r: f64,
    pub c_sb: f64,
    pub kappa0: f64,
    pub k_cond: f64,
    pub chi: f64,
    pub solve_tol: f64,
    pub newton_heat: f64,
    pub newton_cell: f64,
    pub dt_fixed: f64,
    pub dt_cap: f64,
    pub mg_omega: f64,
    pub inner_tol: f64,
    pub reserved_d: [f64; 2],
    pub k1e: f64,
    pub k2e: f64,
    pub k1n: f64,
    pub k2n: f64,
    pub kappa_dust: f64,
    pub t_dust: f64,
    pub sigma_hold: f64,
    pub eta_hold: f64,
    pub r_hold: f64,
    pub m_tov: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct sr_dt_report {
    pub dt: f64,
    pub dt_next: f64,
    pub steps: u64,
    pub sim_time: f64,
    pub non_finite: i32,
    pub nf_channel: i32,
    pub nf_cell: i64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct sr_heat_report {
    pub dt: f64,
    pub passes: u32,
    pub rounds: u32,
    pub refinements: u32,
    pub converged: u32,
    pub delta: f64,
    pub radiated: f64,
    pub rel_residual: f64,
    pub fallback_used: u32,
    pub precond: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct sr_box_report {
    pub x0: u32,
    pub y0: u32,
    pub w: u32,
    pub h: u32,
    pub fft_w: u32,
    pub fft_h: u32,
    pub fits: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct sr_cost {
    pub steps: u32,
    pub pad: u32,
    pub gravity_ms: f64,
    pub hydro_ms: f64,
    pub heat_ms: f64,
    pub floors_ms: f64,
    pub dt_ms: f64,
    pub total_ms: f64,
    pub hydro_update_ms: f64,
    pub hydro_update_launches: u32,
    pub pad2: u32,
    pub kernel_launches: u64,
}

#[repr(C)]
pub struct sr_ctx {
    _opaque: [u8; 0],
}
#[repr(C)]
pub struct sr_learner {
    _opaque: [u8; 0],
}
#[repr(C)]
pub struct sr_batch {
    _opaque: [u8; 0],
}

extern "C" {
    pub fn sr_config_default(cfg: *mut sr_config);
    pub fn sr_abi_version() -> u32;
    pub fn sr_create(cfg: *const sr_config, out: *mut *mut sr_ctx) -> sr_status;
    pub fn sr_destroy(ctx: *mut sr_ctx);
    pub fn sr_upload(ctx: *mut sr_ctx, planes: *const f32, nplanes: u32) -> sr_status;
    pub fn sr_readback(ctx: *mut sr_ctx, planes: *mut f32, nplanes: u32) -> sr_status;
    pub fn sr_upload_held(ctx: *mut sr_ctx, mask: *const u32) -> sr_status;
    pub fn sr_read_box(ctx: *mut sr_ctx, out: *mut sr_box_report) -> sr_status;
    pub fn sr_read_held(ctx: *mut sr_ctx, mask: *mut u32) -> sr_status;
    pub fn sr_upload_opacity(ctx: *mut sr_ctx, kappa: *const f32) -> sr_status;
    pub fn sr_step(ctx: *mut sr_ctx, steps: u32) -> sr_status;
    pub fn sr_read_dt(ctx: *mut sr_ctx, out: *mut sr_dt_report) -> sr_status;
    pub fn sr_read_heat(ctx: *mut sr_ctx, out: *mut sr_heat_report) -> sr_status;
    pub fn sr_gravity_field(ctx: *mut sr_ctx, gx: *mut f32, gy: *mut f32, phi: *mut f32) -> sr_status;
    pub fn sr_heat_flux(ctx: *mut sr_ctx, fx: *mut f32, fy: *mut f32) -> sr_status;
    pub fn sr_set_clock(ctx: *mut sr_ctx, steps: u64, sim_time: f64, dt: f64, dt_next: f64) -> sr_status;
    pub fn sr_read_heat_rate(ctx: *mut sr_ctx, rate: *mut f32) -> sr_status;
    pub fn sr_set_heat_rate(ctx: *mut sr_ctx, rate: *const f32) -> sr_status;
    pub fn sr_read_side_flux(ctx: *mut sr_ctx, fx: *mut f32, fy: *mut f32) -> sr_status;
    pub fn sr_set_side_flux(ctx: *mut sr_ctx, fx: *const f32, fy: *const f32) -> sr_status;
    pub fn sr_set_edge_mode(ctx: *mut sr_ctx, edge: u32) -> sr_status;
    pub fn sr_set_heat_precond(ctx: *mut sr_ctx, precond: u32) -> sr_status;
    pub fn sr_set_heat_limits(ctx: *mut sr_ctx, max_passes: u32, max_rounds: u32) -> sr_status;
    pub fn sr_set_timing(ctx: *mut sr_ctx, on: i32) -> sr_status;
    pub fn sr_read_cost(ctx: *mut sr_ctx, out: *mut sr_cost) -> sr_status;
    pub fn sr_heat_first_solve(ctx: *mut sr_ctx, dt: f64, precond: u32, ms: *mut f64, rounds: *mut u32,
                               rel_residual: *mut f64, x: *mut f64, fallback: *mut u32) -> sr_status;
    pub fn sr_time_smoother(ctx: *mut sr_ctx, reps: u32, pre_ms: *mut f64, post_ms: *mut f64) -> sr_status;
    pub fn sr_learner_create(crop: u32, capacity: u32, seed: u64, out: *mut *mut sr_learner) -> sr_status;
    pub fn sr_learner_destroy(learner: *mut sr_learner);
    pub fn sr_learner_param_count() -> u32;
    pub fn sr_learner_get_params(learner: *mut sr_learner, theta: *mut f32) -> sr_status;
    pub fn sr_learner_set_params(learner: *mut sr_learner, theta: *const f32) -> sr_status;
    pub fn sr_learner_collect(learner: *mut sr_learner, ctx: *mut sr_ctx, dt: f64, crops: u32, seed: u64,
                              samples: *mut u32) -> sr_status;
    pub fn sr_learner_train(learner: *mut sr_learner, iterations: u32, batch: u32, lr: f64, seed: u64,
                            loss: *mut f64) -> sr_status;
    pub fn sr_learner_loss_grad(learner: *mut sr_learner, feats: *const f32, target: *const f32, n: u32,
                                loss: *mut f64, grad: *mut f32, out: *mut f32) -> sr_status;
    pub fn sr_attach_learner(ctx: *mut sr_ctx, learner: *mut sr_learner) -> sr_status;
    pub fn sr_batch_create(cfgs: *const sr_config, count: u32, threads: u32, out: *mut *mut sr_batch) -> sr_status;
    pub fn sr_batch_destroy(b: *mut sr_batch);
    pub fn sr_batch_upload(b: *mut sr_batch, index: u32, planes: *const f32, kappa: *const f32) -> sr_status;
    pub fn sr_batch_step(b: *mut sr_batch, steps: u32, device_ms: *mut f64) -> sr_status;
    pub fn sr_batch_readback(b: *mut sr_batch, index: u32, planes: *mut f32) -> sr_status;
    pub fn sr_batch_ctx(b: *mut sr_batch, index: u32) -> *mut sr_ctx;
    pub fn sr_gravity_solve_static(cfg: *const sr_config, sigma: *const f32, phi: *mut f32, gx: *mut f32,
                                   gy: *mut f32, stream: *mut c_void) -> sr_status;
    pub fn sr_last_error(ctx: *const sr_ctx) -> *const c_char;
}

/// A refused or failed call: the status and the library's message.
#[derive(Debug, Clone)]
pub struct Error {
    pub status: sr_status,
    pub message: String,
}

impl std::fmt::Display for Error {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        write!(f, "status {}: {}", self.status, self.message)
    }
}

impl std::error::Error for Error {}

fn last_error(ctx: *const sr_ctx) -> String {
    unsafe {
        let p = sr_last_error(ctx);
        if p.is_null() { String::new() } else { CStr::from_ptr(p).to_string_lossy().into_owned() }
    }
}

/// The library's defaults: physics.json's shipped constants and the reference's scheme.
pub fn default_config() -> sr_config {
    let mut c = sr_config::default();
    unsafe { sr_config_default(&mut c) };
    c
}

/// One world on the GPU: the reference's `Step` + `State` pair over the C ABI. Not `Sync`: one host thread at a time
/// (the reference's `Step` is `!Sync` too).
pub struct Step {
    ctx: *mut sr_ctx,
    cfg: sr_config,
}

impl Step {
    /// `Step::with_heat` / `with_passes` (step/mod.rs:399-527): validates the world and allocates its buffers.
    pub fn new(cfg: &sr_config) -> Result<Step, Error> {
        let mut ctx = std::ptr::null_mut();
        let st = unsafe { sr_create(cfg, &mut ctx) };
        if st != SR_OK {
            return Err(Error { status: st, message: last_error(std::ptr::null()) });
        }
        Ok(Step { ctx, cfg: *cfg })
    }

    fn check(&self, st: sr_status) -> Result<(), Error> {
        if st == SR_OK { Ok(()) } else { Err(Error { status: st, message: last_error(self.ctx) }) }
    }

    fn plane_len(&self) -> usize {
        self.cfg.width as usize * self.cfg.height as usize
    }

    /// `State::upload` (state.rs:251): the context's canonical channel-major f32 planes (4, or 14 in reference mode).
    pub fn upload(&mut self, planes: &[f32]) -> Result<(), Error> {
        let nc = self.cfg.channels as usize;
        assert_eq!(planes.len(), nc * self.plane_len(), "one plane of width x height per channel");
        self.check(unsafe { sr_upload(self.ctx, planes.as_ptr(), nc as u32) })
    }

    /// `State::upload_held` (state.rs:198-211): the hold's mask, one word per cell (reference mode).
    pub fn upload_held(&mut self, mask: &[u32]) -> Result<(), Error> {
        assert_eq!(mask.len(), self.plane_len(), "one word per cell");
        self.check(unsafe { sr_upload_held(self.ctx, mask.as_ptr()) })
    }

    /// `State::read_held` (state.rs:213-250).
    pub fn read_held(&mut self, mask: &mut [u32]) -> Result<(), Error> {
        assert_eq!(mask.len(), self.plane_len(), "one word per cell");
        self.check(unsafe { sr_read_held(self.ctx, mask.as_mut_ptr()) })
    }

    pub fn upload_opacity(&mut self, kappa: &[f32]) -> Result<(), Error> {
        assert_eq!(kappa.len(), self.plane_len(), "one plane of width x height");
        self.check(unsafe { sr_upload_opacity(self.ctx, kappa.as_ptr()) })
    }

    /// `Step::restore` (step/latch.rs:493-510): the next step's index, the sim time, Δt_n and the next Δt.
    pub fn set_clock(&mut self, steps: u64, sim_time: f64, dt: f64, dt_next: f64) -> Result<(), Error> {
        self.check(unsafe { sr_set_clock(self.ctx, steps, sim_time, dt, dt_next) })
    }

    /// `Step::heat_rate` (step/heat.rs:550-565): each cell's P5 rate of the last step.
    pub fn heat_rate(&mut self, rate: &mut [f32]) -> Result<(), Error> {
        assert_eq!(rate.len(), self.plane_len(), "one plane of width x height");
        self.check(unsafe { sr_read_heat_rate(self.ctx, rate.as_mut_ptr()) })
    }

    /// `Step::set_heat_rate` (step/heat.rs:566-582): a dump's rate, or zeros for None.
    pub fn set_heat_rate(&mut self, rate: Option<&[f32]>) -> Result<(), Error> {
        let ptr = match rate {
            Some(r) => {
                assert_eq!(r.len(), self.plane_len(), "one plane of width x height");
                r.as_ptr()
            }
            None => std::ptr::null(),
        };
        self.check(unsafe { sr_set_heat_rate(self.ctx, ptr) })
    }

    /// `Step::side_flux` (step/heat.rs:584-589), read back: the cell-centred F the next P4 pushes with.
    pub fn side_flux(&mut self, fx: &mut [f32], fy: &mut [f32]) -> Result<(), Error> {
        assert!(fx.len() == self.plane_len() && fy.len() == self.plane_len(), "one plane of width x height each");
        self.check(unsafe { sr_read_side_flux(self.ctx, fx.as_mut_ptr(), fy.as_mut_ptr()) })
    }

    /// `load_dump`'s write of F into the step's side flux (dump.rs:404-407).
    pub fn set_side_flux(&mut self, fx: &[f32], fy: &[f32]) -> Result<(), Error> {
        assert!(fx.len() == self.plane_len() && fy.len() == self.plane_len(), "one plane of width x height each");
        self.check(unsafe { sr_set_side_flux(self.ctx, fx.as_ptr(), fy.as_ptr()) })
    }

    /// `Step::run` (step/mod.rs:703-718).
    pub fn run(&mut self, steps: u32) -> Result<(), Error> {
        self.check(unsafe { sr_step(self.ctx, steps) })
    }

    /// `State::readback` (state.rs:273).
    pub fn readback(&mut self, planes: &mut [f32]) -> Result<(), Error> {
        let nc = self.cfg.channels as usize;
        assert_eq!(planes.len(), nc * self.plane_len(), "one plane of width x height per channel");
        self.check(unsafe { sr_readback(self.ctx, planes.as_mut_ptr(), nc as u32) })
    }

    /// `Step::read_dt` (step/dt.rs:173).
    pub fn read_dt(&mut self) -> Result<sr_dt_report, Error> {
        let mut r = sr_dt_report::default();
        self.check(unsafe { sr_read_dt(self.ctx, &mut r) })?;
        Ok(r)
    }

    /// `Step::read_heat` (step/heat.rs:499-512).
    pub fn read_heat(&mut self) -> Result<sr_heat_report, Error> {
        let mut r = sr_heat_report::default();
        self.check(unsafe { sr_read_heat(self.ctx, &mut r) })?;
        Ok(r)
    }

    pub fn raw(&mut self) -> *mut sr_ctx {
        self.ctx
    }
}

impl Drop for Step {
    fn drop(&mut self) {
        unsafe { sr_destroy(self.ctx) };
    }
}
