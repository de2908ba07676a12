//! A safe owner of one device grid (`wf_handle`): created and destroyed with
//! it, every call's status turned into a `Result`.  The reference's
//! `engine::run` (src/engine.rs:653-661) is re-implemented on top of this by
//! the maintainer's wrapper: set materials, CPML profiles, source values and
//! probe tables once, then `step`, read the probe sums and the snapshots.

use crate::*;
use std::ffi::{CStr, CString};
use std::ptr;

/// A failed call: the status and the library's message for it.
#[derive(Debug, Clone)]
pub struct Error {
    pub status: wf_status,
    pub message: String,
}

impl std::fmt::Display for Error {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        write!(f, "wavefront_gpu error {}: {}", self.status, self.message)
    }
}

impl std::error::Error for Error {}

impl From<Error> for std::io::Error {
    fn from(e: Error) -> Self {
        std::io::Error::new(std::io::ErrorKind::Other, e)
    }
}

/// One grid on one device (not thread-safe: one handle per host thread).
pub struct Handle {
    h: *mut wf_handle,
    cells: usize,
}

impl Handle {
    fn check(&self, st: wf_status) -> Result<(), Error> {
        if st == WF_OK {
            return Ok(());
        }
        let msg = unsafe { CStr::from_ptr(wf_last_error(self.h)) }.to_string_lossy().into_owned();
        Err(Error { status: st, message: msg })
    }

    /// A grid of nx x ny x nz voxels (multiples of 8) with zero-field
    /// boundaries, the exact arithmetic and FP32 storage on `device`.
    pub fn new(nx: i32, ny: i32, nz: i32, device: i32) -> Result<Handle, Error> {
        let d = wf_grid_desc {
            nx,
            ny,
            nz,
            boundary: [WF_BOUNDARY_ZERO; 3],
            arith: WF_ARITH_EXACT,
            kernel: WF_KERNEL_AUTO,
            precision: WF_PREC_F32,
            device,
            stream: ptr::null_mut(),
        };
        Handle::with_desc(&d)
    }

    pub fn with_desc(d: &wf_grid_desc) -> Result<Handle, Error> {
        let mut h = ptr::null_mut();
        let st = unsafe { wf_create(d, &mut h) };
        if st != WF_OK {
            let msg = unsafe { CStr::from_ptr(wf_last_error(ptr::null())) }.to_string_lossy().into_owned();
            return Err(Error { status: st, message: msg });
        }
        let cells = d.nx as usize * d.ny as usize * d.nz as usize;
        Ok(Handle { h, cells })
    }

    /// MaterialGrid bytes (z, y, x order) and the 256-entry Q16.16 table.
    pub fn set_materials(&mut self, ids: &[u8], table_q16: &[[i32; 4]; 256]) -> Result<(), Error> {
        assert_eq!(ids.len(), self.cells, "one material id per voxel");
        self.check(unsafe { wf_set_materials(self.h, ids.as_ptr(), table_q16.as_ptr()) })
    }

    /// One axis's CPML profile (b, a, 1/kappa over the axis's n positions).
    pub fn set_pml(&mut self, axis: i32, thickness: i32, b: &[f32], a: &[f32], inv_kappa: &[f32])
                   -> Result<(), Error> {
        assert!(b.len() == a.len() && a.len() == inv_kappa.len());
        self.check(unsafe { wf_set_pml(self.h, axis, thickness, b.as_ptr(), a.as_ptr(), inv_kappa.as_ptr()) })
    }

    /// A soft point source with its per-step values (amplitude * w((s+1) dt));
    /// returns its index.
    pub fn add_source(&mut self, x: i32, y: i32, z: i32, comp: i32, values: &[f32]) -> Result<i32, Error> {
        let mut idx = -1;
        self.check(unsafe {
            wf_add_source(self.h, x, y, z, comp, 0, values.as_ptr(), values.len() as c_int, &mut idx)
        })?;
        Ok(idx)
    }

    /// A DFT probe with its twiddle tables ([nsteps][nfreq] each); returns
    /// its index.
    pub fn add_probe(&mut self, x: i32, y: i32, z: i32, comp: i32, nfreq: i32, cos_tab: &[f64],
                     sin_tab: &[f64], first_step: i32) -> Result<i32, Error> {
        assert_eq!(cos_tab.len(), sin_tab.len());
        let nsteps = (cos_tab.len() / nfreq.max(1) as usize) as c_int;
        let mut idx = -1;
        self.check(unsafe {
            wf_add_probe(self.h, x, y, z, comp, nfreq, cos_tab.as_ptr(), sin_tab.as_ptr(), nsteps,
                         first_step, 0, &mut idx)
        })?;
        Ok(idx)
    }

    /// Enqueues n full steps (H, E, sources, probes) on the handle's stream.
    pub fn step(&mut self, n: i32) -> Result<(), Error> {
        self.check(unsafe { wf_step(self.h, n) })
    }

    /// Waits for the enqueued steps; reports latched device errors.
    pub fn sync(&mut self) -> Result<(), Error> {
        self.check(unsafe { wf_sync(self.h) })
    }

    /// (sum cos, sum sin, samples) of probe p.
    pub fn probe_sums(&mut self, p: i32, nfreq: usize) -> Result<(Vec<f64>, Vec<f64>, u64), Error> {
        let (mut c, mut s, mut n) = (vec![0f64; nfreq], vec![0f64; nfreq], 0u64);
        self.check(unsafe { wf_probe_sums(self.h, p, c.as_mut_ptr(), s.as_mut_ptr(), &mut n) })?;
        Ok((c, s, n))
    }

    /// The state in the reference's FieldBlock byte order (24 bytes a voxel),
    /// for the snapshot writer.
    pub fn download_blocks(&mut self, out: &mut [u8]) -> Result<(), Error> {
        assert_eq!(out.len(), self.cells * 24);
        self.check(unsafe { wf_download_blocks(self.h, out.as_mut_ptr().cast()) })
    }

    /// Scene text through the device voxelizer (the reference's rules and
    /// messages); fills the table's registered materials.
    pub fn set_scene(&mut self, text: &str, dt: f32, dx: f32, table_q16: &mut [[i32; 4]; 256])
                     -> Result<i32, Error> {
        let t = CString::new(text).expect("scene text without NUL bytes");
        let mut n = 0;
        self.check(unsafe { wf_set_scene(self.h, t.as_ptr(), dt, dx, table_q16.as_mut_ptr(), &mut n) })?;
        Ok(n)
    }

    pub fn raw(&self) -> *mut wf_handle {
        self.h
    }
}

impl Drop for Handle {
    fn drop(&mut self) {
        unsafe {
            wf_destroy(self.h);
        }
    }
}
