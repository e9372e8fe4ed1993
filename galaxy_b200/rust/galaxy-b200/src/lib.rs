//! `GpuLbvhB200`, `GpuStaleTreeB200`, `GpuGravitySphB200` and `GpuResidentB200`: galaxy's
//! gravity-solver interface over libgalaxy_b200 (a B200 LBVH Barnes-Hut). `GpuLbvhB200`
//! implements `ForceSolver` (core/src/traits.rs) and drops in beside `Lbvh`, `BarnesHut`
//! and `GpuLbvhFused`; `GpuStaleTreeB200` plays `TreeGravity`'s stale-tree role for
//! individual time steps; `GpuGravitySphB200` plays `GravitySph<Lbvh>`
//! (solvers/src/sph/gravity_sph.rs); `GpuResidentB200` mirrors `GpuResidentLeapfrog`'s
//! upload / step_many / snapshot and, from `new_with_sph`, its gas mode.
//!
//! Written against include/galaxy_b200.h; DVec3 is three f64 (`#[repr(C)]`-compatible
//! in glam), so `&[DVec3]` is passed as `*const f64` with no copy.

use galaxy_core::{DVec3, ForceSolver, SfFields, State};
use galaxy_solvers::sph::{DensityConfig, Eos, HydroParams};
use std::ffi::CStr;
use std::os::raw::{c_char, c_int};

#[repr(C)]
#[derive(Clone, Copy, Default)]
pub struct GxOptions {
    pub struct_size: u32,
    pub precision: u32,
    pub multipole: u32,
    pub flags: u32,
    pub device: i32,
    pub walk_block: u32,
    pub walk_ctas_per_sm: u32,
    pub walk_group: u32,
    pub radix_bits: u32,
}

#[repr(C)]
pub struct GxHandle {
    _private: [u8; 0],
}

/// `gx_sph_params`: HydroParams + DensityConfig as the C ABI takes them.
#[repr(C)]
#[derive(Clone, Copy, Default)]
pub struct GxSphParams {
    pub n_ngb: f64,
    pub h_tol_rel: f64,
    pub eos: c_int,
    pub warm_start: c_int,
    pub c_s: f64,
    pub gamma: f64,
    pub alpha: f64,
    pub beta: f64,
    pub visc_eps2: f64,
}

impl GxSphParams {
    /// The reference's parameters (forces.rs:64-87, density.rs:33-51); h warm-started
    /// across evaluations as GravitySph does.
    pub fn from_reference(hydro: &HydroParams, density: &DensityConfig) -> Self {
        let (eos, c_s, gamma) = match hydro.eos {
            Eos::Isothermal { c_s } => (0, c_s, 5.0 / 3.0),
            Eos::Adiabatic { gamma } => (1, 0.0, gamma),
        };
        GxSphParams { n_ngb: density.n_ngb, h_tol_rel: density.h_tol_rel, eos, warm_start: 1, c_s, gamma,
                      alpha: hydro.alpha, beta: hydro.beta, visc_eps2: hydro.visc_eps2 }
    }
}

extern "C" {
    fn gx_sph_enable(h: *mut GxHandle, p: *const GxSphParams) -> c_int;
    fn gx_upload_species(h: *mut GxHandle, n: usize, pos: *const f64, vel: *const f64, mass: *const f64,
                         kind: *const u8, u: *const f64) -> c_int;
    fn gx_gas_count(h: *const GxHandle, n_gas: *mut usize) -> c_int;
    fn gx_snapshot_gas_density(h: *mut GxHandle, gas_idx: *mut u32, rho: *mut f64, hsml: *mut f64) -> c_int;
    fn gx_snapshot_gas_accel(h: *mut GxHandle, acc: *mut f64, dudt: *mut f64) -> c_int;
    fn gx_snapshot_accel(h: *mut GxHandle, acc: *mut f64) -> c_int;
    fn gx_min_stable_dt(h: *mut GxHandle, c_cfl: f64, out: *mut f64) -> c_int;
    fn gx_snapshot_gas_dt(h: *mut GxHandle, c_cfl: f64, dt: *mut f64) -> c_int;
    fn gx_sph_accelerations(h: *mut GxHandle, n: usize, pos: *const f64, vel: *const f64, mass: *const f64,
                            kind: *const u8, u: *const f64, acc: *mut f64) -> c_int;
    fn gx_sph_accelerations_active(h: *mut GxHandle, n: usize, pos: *const f64, vel: *const f64,
                                   mass: *const f64, kind: *const u8, u: *const f64, n_active: usize,
                                   active: *const u32, acc: *mut f64) -> c_int;
    fn gx_sph_accel_and_dudt_active(h: *mut GxHandle, n: usize, pos: *const f64, vel: *const f64,
                                    mass: *const f64, kind: *const u8, u: *const f64, n_active: usize,
                                    active: *const u32, acc: *mut f64, dudt: *mut f64) -> c_int;
    fn gx_sph_sf_fields(h: *mut GxHandle, n: usize, pos: *const f64, vel: *const f64, mass: *const f64,
                        kind: *const u8, rho: *mut f64, div: *mut f64) -> c_int;
    fn gx_sph_accel_and_dudt(h: *mut GxHandle, n: usize, pos: *const f64, vel: *const f64, mass: *const f64,
                             kind: *const u8, u: *const f64, acc: *mut f64, dudt: *mut f64) -> c_int;
    fn gx_sph_max_stable_dt(h: *mut GxHandle, n: usize, pos: *const f64, vel: *const f64, mass: *const f64,
                            kind: *const u8, u: *const f64, c_cfl: f64, dt: *mut f64, min: *mut f64) -> c_int;
    fn gx_sph_coupled_pairs(h: *mut GxHandle, n: usize, pos: *const f64, mass: *const f64, kind: *const u8,
                            pairs: *mut u64, cap: usize, count: *mut usize) -> c_int;
}

extern "C" {
    fn gx_create(g: f64, softening: f64, theta: f64, opt: *const GxOptions, out: *mut *mut GxHandle) -> c_int;
    fn gx_destroy(h: *mut GxHandle);
    fn gx_last_error(h: *const GxHandle) -> *const c_char;
    fn gx_accelerations(h: *mut GxHandle, n: usize, pos: *const f64, mass: *const f64, acc: *mut f64) -> c_int;
    fn gx_accelerations_active(
        h: *mut GxHandle,
        n: usize,
        pos: *const f64,
        mass: *const f64,
        n_active: usize,
        active: *const u32,
        acc: *mut f64,
    ) -> c_int;
    fn gx_potential_energy(h: *mut GxHandle, n: usize, pos: *const f64, mass: *const f64, out: *mut f64) -> c_int;
    fn gx_rebuild_gravity_cache(h: *mut GxHandle, n: usize, pos: *const f64, mass: *const f64) -> c_int;
    fn gx_gravity_active_cached(
        h: *mut GxHandle,
        n: usize,
        pos: *const f64,
        mass: *const f64,
        n_active: usize,
        active: *const u32,
        acc: *mut f64,
    ) -> c_int;
    fn gx_upload(h: *mut GxHandle, n: usize, pos: *const f64, vel: *const f64, mass: *const f64) -> c_int;
    fn gx_step_many(h: *mut GxHandle, dt: f64, steps: u64) -> c_int;
    fn gx_snapshot(h: *mut GxHandle, pos: *mut f64, vel: *mut f64) -> c_int;
    fn gx_time(h: *const GxHandle, t: *mut f64) -> c_int;
}

/// Error of a libgalaxy_b200 call: the status code and the library's message.
#[derive(Debug)]
pub struct GxError {
    pub code: i32,
    pub message: String,
}

fn err(h: *const GxHandle, code: c_int) -> GxError {
    let msg = unsafe { CStr::from_ptr(gx_last_error(h)) }.to_string_lossy().into_owned();
    GxError { code, message: msg }
}

fn as_f64(v: &[DVec3]) -> *const f64 {
    debug_assert_eq!(std::mem::size_of::<DVec3>(), 24);
    v.as_ptr() as *const f64
}

/// Drop-in `ForceSolver` (the role of `GpuLbvhFused`): host state in, accelerations out.
pub struct GpuLbvhB200 {
    h: *mut GxHandle,
    pub g: f64,
    pub softening: f64,
}

impl GpuLbvhB200 {
    /// `precision`: 0 = FP32 walk (default), 1 = FP64 (bit-identical to `Lbvh`).
    pub fn new(g: f64, softening: f64, theta: f64, precision: u32) -> Result<Self, GxError> {
        let opt = GxOptions { struct_size: std::mem::size_of::<GxOptions>() as u32, precision, device: -1, ..Default::default() };
        let mut h = std::ptr::null_mut();
        let rc = unsafe { gx_create(g, softening, theta, &opt, &mut h) };
        if rc != 0 {
            return Err(err(std::ptr::null(), rc));
        }
        Ok(Self { h, g, softening })
    }
}

impl Drop for GpuLbvhB200 {
    fn drop(&mut self) {
        unsafe { gx_destroy(self.h) }
    }
}

impl ForceSolver for GpuLbvhB200 {
    fn accelerations(&mut self, state: &State, acc: &mut [DVec3]) {
        let n = state.len();
        assert_eq!(acc.len(), n, "acc length must match particle count");
        let rc = unsafe {
            gx_accelerations(self.h, n, as_f64(&state.pos), state.mass.as_ptr(), acc.as_mut_ptr() as *mut f64)
        };
        // A device failure here is a lost GPU, as in GpuLbvhFused: panic rather than corrupt state.
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.h, rc));
    }

    // The individual-timestep path: walk the tree for the active targets only; each gets
    // the acceleration `accelerations` would give it (rows outside `active` untouched).
    fn accelerations_active(&mut self, state: &State, active: &[usize], acc: &mut [DVec3]) {
        let n = state.len();
        assert_eq!(acc.len(), n, "acc length must match particle count");
        let idx: Vec<u32> = active.iter().map(|&i| u32::try_from(i).expect("active index fits u32")).collect();
        let rc = unsafe {
            gx_accelerations_active(
                self.h,
                n,
                as_f64(&state.pos),
                state.mass.as_ptr(),
                idx.len(),
                idx.as_ptr(),
                acc.as_mut_ptr() as *mut f64,
            )
        };
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.h, rc));
    }

    // Lbvh caches nothing between calls: the stale-tree walk is a fresh active pass.
    fn gravity_active_cached(&mut self, state: &State, active: &[usize], acc: &mut [DVec3]) {
        self.accelerations_active(state, active, acc);
    }

    fn potential_energy(&self, state: &State) -> f64 {
        let mut u = 0.0;
        let rc = unsafe { gx_potential_energy(self.h, state.len(), as_f64(&state.pos), state.mass.as_ptr(), &mut u) };
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.h, rc));
        u
    }
}

/// The stale-tree active walk of `TreeGravity` (solvers/src/barnes_hut.rs:647-711) over the
/// LBVH: `rebuild_gravity_cache` freezes the tree at the block-start state and
/// `gravity_active_cached` walks it at the current positions (leaf sources current,
/// internal aggregates frozen). Fresh passes run on a second handle and leave the cache.
pub struct GpuStaleTreeB200 {
    cache: *mut GxHandle,
    fresh: GpuLbvhB200,
    cached: bool,
}

impl GpuStaleTreeB200 {
    pub fn new(g: f64, softening: f64, theta: f64, precision: u32) -> Result<Self, GxError> {
        let fresh = GpuLbvhB200::new(g, softening, theta, precision)?;
        let opt = GxOptions { struct_size: std::mem::size_of::<GxOptions>() as u32, precision, device: -1, ..Default::default() };
        let mut h = std::ptr::null_mut();
        let rc = unsafe { gx_create(g, softening, theta, &opt, &mut h) };
        if rc != 0 {
            return Err(err(std::ptr::null(), rc));
        }
        Ok(Self { cache: h, fresh, cached: false })
    }
}

impl ForceSolver for GpuStaleTreeB200 {
    fn accelerations(&mut self, state: &State, acc: &mut [DVec3]) {
        self.fresh.accelerations(state, acc);
    }

    fn rebuild_gravity_cache(&mut self, state: &State) {
        let rc = unsafe { gx_rebuild_gravity_cache(self.cache, state.len(), as_f64(&state.pos), state.mass.as_ptr()) };
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.cache, rc));
        self.cached = !state.is_empty(); // an empty state has no tree: later walks do nothing
    }

    fn gravity_active_cached(&mut self, state: &State, active: &[usize], acc: &mut [DVec3]) {
        assert_eq!(acc.len(), state.len(), "acc length must match particle count");
        if !self.cached {
            return; // never rebuilt: nothing to walk, as TreeGravity
        }
        let idx: Vec<u32> = active.iter().map(|&i| u32::try_from(i).expect("active index fits u32")).collect();
        let rc = unsafe {
            gx_gravity_active_cached(
                self.cache,
                state.len(),
                as_f64(&state.pos),
                state.mass.as_ptr(),
                idx.len(),
                idx.as_ptr(),
                acc.as_mut_ptr() as *mut f64,
            )
        };
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.cache, rc));
    }

    fn potential_energy(&self, state: &State) -> f64 {
        self.fresh.potential_energy(state)
    }
}

impl Drop for GpuStaleTreeB200 {
    fn drop(&mut self) {
        unsafe { gx_destroy(self.cache) }
    }
}

/// `GravitySph<Lbvh>` (solvers/src/sph/gravity_sph.rs:172-207): gravity on every
/// particle, density, smoothing lengths and the hydro force on the gas rows, h
/// warm-started across calls while the gas count holds.
pub struct GpuGravitySphB200 {
    h: *mut GxHandle,
}

impl GpuGravitySphB200 {
    pub fn new(g: f64, softening: f64, theta: f64, hydro: HydroParams, density: DensityConfig)
               -> Result<Self, GxError> {
        let mut h = std::ptr::null_mut();
        let rc = unsafe { gx_create(g, softening, theta, std::ptr::null(), &mut h) };
        if rc != 0 {
            return Err(err(std::ptr::null(), rc));
        }
        let p = GxSphParams::from_reference(&hydro, &density);
        let rc = unsafe { gx_sph_enable(h, &p) };
        if rc != 0 {
            let e = err(h, rc);
            unsafe { gx_destroy(h) };
            return Err(e);
        }
        Ok(Self { h })
    }
}

impl ForceSolver for GpuGravitySphB200 {
    fn accelerations(&mut self, state: &State, acc: &mut [DVec3]) {
        let n = state.len();
        assert_eq!(acc.len(), n, "acc length must match particle count");
        // Species is #[repr(u8)] (Collisionless = 0, Gas = 1): the column crosses as bytes.
        let rc = unsafe {
            gx_sph_accelerations(self.h, n, as_f64(&state.pos), as_f64(&state.vel), state.mass.as_ptr(),
                                 state.kind.as_ptr() as *const u8, state.u.as_ptr(), acc.as_mut_ptr() as *mut f64)
        };
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.h, rc));
    }

    fn accel_and_dudt(&mut self, state: &State, acc: &mut [DVec3], dudt: &mut [f64]) {
        let n = state.len();
        assert_eq!(acc.len(), n, "acc length must match particle count");
        assert_eq!(dudt.len(), n, "dudt length must match particle count");
        let rc = unsafe {
            gx_sph_accel_and_dudt(self.h, n, as_f64(&state.pos), as_f64(&state.vel), state.mass.as_ptr(),
                                  state.kind.as_ptr() as *const u8, state.u.as_ptr(), acc.as_mut_ptr() as *mut f64,
                                  dudt.as_mut_ptr())
        };
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.h, rc));
    }

    fn accelerations_active(&mut self, state: &State, active: &[usize], acc: &mut [DVec3]) {
        let n = state.len();
        assert_eq!(acc.len(), n, "acc length must match particle count");
        let idx: Vec<u32> = active.iter().map(|&i| i as u32).collect();
        let rc = unsafe {
            gx_sph_accelerations_active(self.h, n, as_f64(&state.pos), as_f64(&state.vel), state.mass.as_ptr(),
                                        state.kind.as_ptr() as *const u8, state.u.as_ptr(), idx.len(), idx.as_ptr(),
                                        acc.as_mut_ptr() as *mut f64)
        };
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.h, rc));
    }

    fn accel_and_dudt_active(&mut self, state: &State, active: &[usize], acc: &mut [DVec3], dudt: &mut [f64]) {
        let n = state.len();
        assert_eq!(acc.len(), n, "acc length must match particle count");
        assert_eq!(dudt.len(), n, "dudt length must match particle count");
        let idx: Vec<u32> = active.iter().map(|&i| i as u32).collect();
        let rc = unsafe {
            gx_sph_accel_and_dudt_active(self.h, n, as_f64(&state.pos), as_f64(&state.vel), state.mass.as_ptr(),
                                         state.kind.as_ptr() as *const u8, state.u.as_ptr(), idx.len(),
                                         idx.as_ptr(), acc.as_mut_ptr() as *mut f64, dudt.as_mut_ptr())
        };
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.h, rc));
    }

    // GravitySph delegates the cache to its gravity solver; Lbvh caches nothing.
    fn rebuild_gravity_cache(&mut self, _state: &State) {}

    // The gravity-ONLY active walk (gravity_sph.rs:329-341): Lbvh's default, a fresh pass,
    // with no hydro added (the driver's |a_grav| for the combined rung dt).
    fn gravity_active_cached(&mut self, state: &State, active: &[usize], acc: &mut [DVec3]) {
        let n = state.len();
        assert_eq!(acc.len(), n, "acc length must match particle count");
        let idx: Vec<u32> = active.iter().map(|&i| u32::try_from(i).expect("active index fits u32")).collect();
        let rc = unsafe {
            gx_accelerations_active(self.h, n, as_f64(&state.pos), state.mass.as_ptr(), idx.len(), idx.as_ptr(),
                                    acc.as_mut_ptr() as *mut f64)
        };
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.h, rc));
    }

    fn potential_energy(&self, state: &State) -> f64 {
        let mut out = 0.0;
        let rc = unsafe { gx_potential_energy(self.h, state.len(), as_f64(&state.pos), state.mass.as_ptr(), &mut out) };
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.h, rc));
        out
    }

    fn max_stable_dt(&self, state: &State) -> f64 {
        let mut m = f64::INFINITY;
        let rc = unsafe {
            gx_sph_max_stable_dt(self.h, state.len(), as_f64(&state.pos), as_f64(&state.vel), state.mass.as_ptr(),
                                 state.kind.as_ptr() as *const u8, state.u.as_ptr(), 1.0, std::ptr::null_mut(), &mut m)
        };
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.h, rc));
        m
    }

    fn max_stable_dt_per_particle(&self, state: &State) -> Vec<f64> {
        let mut dt = vec![f64::INFINITY; state.len()];
        let mut m = f64::INFINITY;
        let rc = unsafe {
            gx_sph_max_stable_dt(self.h, state.len(), as_f64(&state.pos), as_f64(&state.vel), state.mass.as_ptr(),
                                 state.kind.as_ptr() as *const u8, state.u.as_ptr(), 1.0, dt.as_mut_ptr(), &mut m)
        };
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.h, rc));
        dt
    }

    fn sf_fields(&self, state: &State) -> SfFields {
        let n = state.len();
        let (mut rho, mut div_v) = (vec![0.0; n], vec![0.0; n]);
        let rc = unsafe {
            gx_sph_sf_fields(self.h, n, as_f64(&state.pos), as_f64(&state.vel), state.mass.as_ptr(),
                             state.kind.as_ptr() as *const u8, rho.as_mut_ptr(), div_v.as_mut_ptr())
        };
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.h, rc));
        SfFields { rho, div_v }
    }

    fn coupled_pairs(&self, state: &State) -> Vec<(usize, usize)> {
        let n = state.len();
        let mut count = 0usize;
        let mut buf = vec![0u64; 2 * 64 * n.max(1)];
        let mut call = |buf: &mut Vec<u64>, count: &mut usize| unsafe {
            gx_sph_coupled_pairs(self.h, n, as_f64(&state.pos), state.mass.as_ptr(), state.kind.as_ptr() as *const u8,
                                 buf.as_mut_ptr(), buf.len() / 2, count)
        };
        let mut rc = call(&mut buf, &mut count);
        if rc == 0 && 2 * count > buf.len() {
            buf = vec![0u64; 2 * count];
            rc = call(&mut buf, &mut count);
        }
        assert!(rc == 0, "libgalaxy_b200: {:?}", err(self.h, rc));
        (0..count).map(|k| (buf[2 * k] as usize, buf[2 * k + 1] as usize)).collect()
    }
}

impl Drop for GpuGravitySphB200 {
    fn drop(&mut self) {
        unsafe { gx_destroy(self.h) }
    }
}

/// Device-resident KDK stepping (the role of `GpuResidentLeapfrog`).
pub struct GpuResidentB200 {
    h: *mut GxHandle,
    mass: Vec<f64>,
    kind: Vec<galaxy_core::Species>,
    gas_mode: bool,
}

impl GpuResidentB200 {
    pub fn new(g: f64, softening: f64, theta: f64) -> Result<Self, GxError> {
        let mut h = std::ptr::null_mut();
        let rc = unsafe { gx_create(g, softening, theta, std::ptr::null(), &mut h) };
        if rc != 0 {
            return Err(err(std::ptr::null(), rc));
        }
        Ok(Self { h, mass: Vec::new(), kind: Vec::new(), gas_mode: false })
    }

    /// `GpuResidentLeapfrog::new_with_sph` (gpu/src/gpu_resident.rs:1393): gas mode.
    pub fn new_with_sph(g: f64, softening: f64, theta: f64, hydro: HydroParams, density: DensityConfig)
                        -> Result<Self, GxError> {
        let mut s = Self::new(g, softening, theta)?;
        let p = GxSphParams::from_reference(&hydro, &density);
        let rc = unsafe { gx_sph_enable(s.h, &p) };
        if rc != 0 {
            return Err(err(s.h, rc));
        }
        s.gas_mode = true;
        Ok(s)
    }

    pub fn upload(&mut self, state: &State) -> Result<(), GxError> {
        self.mass = state.mass.clone();
        self.kind = state.kind.clone();
        let rc = unsafe {
            if self.gas_mode {
                gx_upload_species(self.h, state.len(), as_f64(&state.pos), as_f64(&state.vel), state.mass.as_ptr(),
                                  state.kind.as_ptr() as *const u8, state.u.as_ptr())
            } else {
                gx_upload(self.h, state.len(), as_f64(&state.pos), as_f64(&state.vel), state.mass.as_ptr())
            }
        };
        if rc != 0 { Err(err(self.h, rc)) } else { Ok(()) }
    }

    fn gas_count(&self) -> usize {
        let mut n = 0usize;
        unsafe { gx_gas_count(self.h, &mut n) };
        n
    }

    /// `snapshot_gas_density` (gpu_resident.rs:1566): (gas_idx, rho, h).
    pub fn snapshot_gas_density(&mut self) -> Result<(Vec<u32>, Vec<f64>, Vec<f64>), GxError> {
        let ng = self.gas_count();
        let (mut idx, mut rho, mut h) = (vec![0u32; ng], vec![0.0; ng], vec![0.0; ng]);
        let rc = unsafe { gx_snapshot_gas_density(self.h, idx.as_mut_ptr(), rho.as_mut_ptr(), h.as_mut_ptr()) };
        if rc != 0 { Err(err(self.h, rc)) } else { Ok((idx, rho, h)) }
    }

    /// `snapshot_gas_accel` (gpu_resident.rs:1593): the hydro acceleration of the gas rows.
    pub fn snapshot_gas_accel(&mut self) -> Result<Vec<DVec3>, GxError> {
        let mut acc = vec![DVec3::ZERO; self.gas_count()];
        let rc = unsafe { gx_snapshot_gas_accel(self.h, acc.as_mut_ptr() as *mut f64, std::ptr::null_mut()) };
        if rc != 0 { Err(err(self.h, rc)) } else { Ok(acc) }
    }

    /// `snapshot_accel` (gpu_resident.rs:1655).
    pub fn snapshot_accel(&mut self) -> Result<Vec<DVec3>, GxError> {
        let mut acc = vec![DVec3::ZERO; self.mass.len()];
        let rc = unsafe { gx_snapshot_accel(self.h, acc.as_mut_ptr() as *mut f64) };
        if rc != 0 { Err(err(self.h, rc)) } else { Ok(acc) }
    }

    /// `min_stable_dt` (gpu_resident.rs:1614): reduced on the device; +inf without gas.
    pub fn min_stable_dt(&mut self, c_cfl: f64) -> Result<f64, GxError> {
        let mut out = f64::INFINITY;
        let rc = unsafe { gx_min_stable_dt(self.h, c_cfl, &mut out) };
        if rc != 0 { Err(err(self.h, rc)) } else { Ok(out) }
    }

    /// `snapshot_gas_dt` (gpu_resident.rs:1632): the per-gas CFL vector.
    pub fn snapshot_gas_dt(&mut self, c_cfl: f64) -> Result<Vec<f64>, GxError> {
        let mut dt = vec![0.0; self.gas_count()];
        if dt.is_empty() {
            return Ok(dt);
        }
        let rc = unsafe { gx_snapshot_gas_dt(self.h, c_cfl, dt.as_mut_ptr()) };
        if rc != 0 { Err(err(self.h, rc)) } else { Ok(dt) }
    }

    pub fn step_many(&mut self, dt: f64, steps: u64) -> Result<(), GxError> {
        let rc = unsafe { gx_step_many(self.h, dt, steps) };
        if rc != 0 { Err(err(self.h, rc)) } else { Ok(()) }
    }

    pub fn snapshot(&mut self) -> Result<State, GxError> {
        let n = self.mass.len();
        let mut pos = vec![DVec3::ZERO; n];
        let mut vel = vec![DVec3::ZERO; n];
        let rc = unsafe { gx_snapshot(self.h, pos.as_mut_ptr() as *mut f64, vel.as_mut_ptr() as *mut f64) };
        if rc != 0 {
            return Err(err(self.h, rc));
        }
        let mut s = State::from_phase_space(pos, vel, self.mass.clone());
        if self.kind.len() == n {
            s.kind = self.kind.clone();
        }
        unsafe { gx_time(self.h, &mut s.time) };
        Ok(s)
    }
}

impl Drop for GpuResidentB200 {
    fn drop(&mut self) {
        unsafe { gx_destroy(self.h) }
    }
}
