//! Drop-in for the two data-parallel paths of cfgable-matmul, computed on an
//! NVIDIA B200 through libcfgmm (the C ABI declared in `include/cfgmm.h`).
//!
//! The public items keep the reference crate's names, module paths and
//! signatures, so a caller switches by changing its dependency:
//!
//! | reference item | here |
//! |---|---|
//! | `MatmulLoops::<T,MC,KC,NC,MR,NR_LANE,LANE>::matmul_loop_parallel_mnk_pack_a` (src/impl_matmul.rs:155-231) | same; `cfgmm_matmul_loop_parallel_mnk_pack_a` |
//! | `impl_matmul::matmul_anyway_full` (src/impl_matmul.rs:234-248) | same; `cfgmm_matmul_anyway_full` |
//! | README's `matmul_loop_macro_mb` (README.md:22-31) | `MatmulLoops::matmul_loop_macro_mb::<MB>`; `cfgmm_matmul_loop_macro_mb` |
//! | `MatmulLoops::matmul_loop_parallel_mnk_pack_a_non0tab::<BLKSIZE>` (src/impl_matmul_non0tab.rs:210-306) | same; `cfgmm_matmul_loop_parallel_mnk_pack_a_non0tab` |
//! | `impl_matmul_non0tab::matmul_anyway_full_non0tab` (src/impl_matmul_non0tab.rs:308-326) | same; `cfgmm_matmul_anyway_full_non0tab` |
//! | `MatmulLoops::aodmao2rho_loop_parallel::<BLKSIZE>` (src/impl_aodmao2rho.rs:171-244) | same; `cfgmm_aodmao2rho_loop_parallel` |
//! | `impl_aodmao2rho::aodmao2rho_anyway` (src/impl_aodmao2rho.rs:247-261) | same; `cfgmm_aodmao2rho_anyway` |
//!
//! Outputs are accumulated into (`C += op(A) op(B)`, `rho += ...`), calls are
//! synchronous and blocking, and every input the reference would panic on
//! (a slice shorter than the index range, `unimplemented!` for the masked
//! GEMM's `transb`) panics here too, with the library's message.  The CPU
//! const generics (`MC`, `KC`, `NC`, `MR`, `NR_LANE`, `LANE`, `BLKSIZE`'s
//! CPU-side constraints) have no meaning on the GPU: the library picks its
//! tiles; `BLKSIZE` keeps its meaning (points per mask block).
//!
//! Beyond the reference: [`Precision`] selects FP64 tensor cores or the
//! Ozaki-style INT8 split precision (max relative error <= 1e-12 against
//! FP64) through the `*_ex` functions, and every wrapper has a `try_` form
//! that returns the status instead of panicking.
#![allow(clippy::too_many_arguments)]

pub mod ffi;

use core::ffi::{c_int, CStr};
use core::marker::PhantomData;

/// Arithmetic of a call.
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum Precision {
    /// FP64 on the DMMA tensor cores.
    Fp64,
    /// Ozaki-style INT8 slices on the tcgen05 tensor cores, FP64 reconstruction.
    OzakiInt8,
}

impl Precision {
    fn code(self) -> c_int {
        match self {
            Precision::Fp64 => ffi::CFGMM_PREC_FP64,
            Precision::OzakiInt8 => ffi::CFGMM_PREC_OZAKI_INT8,
        }
    }
}

/// A nonzero status of the library with its detail message.
#[derive(Clone, Debug, PartialEq, Eq)]
pub struct Error {
    pub status: i32,
    pub message: String,
}

impl core::fmt::Display for Error {
    fn fmt(&self, f: &mut core::fmt::Formatter<'_>) -> core::fmt::Result {
        let what = unsafe { CStr::from_ptr(ffi::cfgmm_status_string(self.status)) };
        write!(f, "cfgmm status {} ({}): {}", self.status, what.to_string_lossy(), self.message)
    }
}

impl std::error::Error for Error {}

fn status(rc: c_int) -> Result<(), Error> {
    if rc == ffi::CFGMM_OK {
        return Ok(());
    }
    let msg = unsafe { CStr::from_ptr(ffi::cfgmm_last_error()) };
    Err(Error { status: rc, message: msg.to_string_lossy().into_owned() })
}

// The reference panics where the library returns a nonzero status.
fn or_panic(r: Result<(), Error>) {
    if let Err(e) = r {
        panic!("{e}");
    }
}

// `&[bool]` is one byte 0/1 per element, the layout `const uint8_t*` reads.
fn tab_ptr(tab: &[bool]) -> *const u8 {
    tab.as_ptr() as *const u8
}

/// The reference's loop type (src/structs.rs:15): the const generics are the
/// CPU blocking of the reference and are accepted for signature
/// compatibility only.
pub struct MatmulLoops<
    T,
    const MC: usize,
    const KC: usize,
    const NC: usize,
    const MR: usize,
    const NR_LANE: usize,
    const LANE: usize,
> {
    _phantom: PhantomData<T>,
}

impl<const MC: usize, const KC: usize, const NC: usize, const MR: usize, const NR_LANE: usize, const LANE: usize>
    MatmulLoops<f64, MC, KC, NC, MR, NR_LANE, LANE>
{
    /// `C[i*ldc + j] += sum_p opA(i,p) opB(p,j)` (src/impl_matmul.rs:155-231).
    pub fn matmul_loop_parallel_mnk_pack_a(
        c: &mut [f64], a: &[f64], b: &[f64], m: usize, n: usize, k: usize, lda: usize,
        ldb: usize, ldc: usize, transa: bool, transb: bool,
    ) {
        or_panic(Self::try_matmul_loop_parallel_mnk_pack_a(c, a, b, m, n, k, lda, ldb, ldc, transa, transb))
    }

    pub fn try_matmul_loop_parallel_mnk_pack_a(
        c: &mut [f64], a: &[f64], b: &[f64], m: usize, n: usize, k: usize, lda: usize,
        ldb: usize, ldc: usize, transa: bool, transb: bool,
    ) -> Result<(), Error> {
        status(unsafe {
            ffi::cfgmm_matmul_loop_parallel_mnk_pack_a(
                c.as_mut_ptr(), c.len(), a.as_ptr(), a.len(), b.as_ptr(), b.len(), m, n, k, lda,
                ldb, ldc, transa as u8, transb as u8,
            )
        })
    }

    /// README.md:22-31's entry point with the L3 block `MB` (ignored: the
    /// library picks its tiles); the same product as above.
    pub fn matmul_loop_macro_mb<const MB: usize>(
        c: &mut [f64], a: &[f64], b: &[f64], m: usize, n: usize, k: usize, lda: usize,
        ldb: usize, ldc: usize, transa: bool, transb: bool,
    ) {
        or_panic(status(unsafe {
            ffi::cfgmm_matmul_loop_macro_mb(
                c.as_mut_ptr(), c.len(), a.as_ptr(), a.len(), b.as_ptr(), b.len(), m, n, k, lda,
                ldb, ldc, transa as u8, transb as u8,
            )
        }))
    }

    /// `C[i,j] += sum_{p: tab[p*ldtab + j/BLKSIZE]} opA(i,p) B[p,j]`
    /// (src/impl_matmul_non0tab.rs:210-306); `transb` panics as the
    /// reference's `unimplemented!` does.
    pub fn matmul_loop_parallel_mnk_pack_a_non0tab<const BLKSIZE: usize>(
        c: &mut [f64], a: &[f64], b: &[f64], m: usize, n: usize, k: usize, lda: usize,
        ldb: usize, ldc: usize, transa: bool, transb: bool, tab: &[bool], ldtab: usize,
    ) {
        or_panic(status(unsafe {
            ffi::cfgmm_matmul_loop_parallel_mnk_pack_a_non0tab(
                c.as_mut_ptr(), c.len(), a.as_ptr(), a.len(), b.as_ptr(), b.len(), m, n, k, lda,
                ldb, ldc, transa as u8, transb as u8, tab_ptr(tab), tab.len(), ldtab, BLKSIZE,
            )
        }))
    }

    /// `rho[s*stride_grid + g] += sum_{u,v active in g's block} ao_lhs[u,g]
    /// D_s[u,v] ao_rhs[v,g]` (src/impl_aodmao2rho.rs:171-244).
    pub fn aodmao2rho_loop_parallel<const BLKSIZE: usize>(
        rhos: &mut [f64], dms: &[f64], ao_lhs: &[f64], ao_rhs: &[f64], strides: [usize; 2],
        shape: [usize; 2], nset: usize, tab: &[bool], ldtab: usize,
    ) {
        or_panic(Self::try_aodmao2rho_loop_parallel::<BLKSIZE>(
            rhos, dms, ao_lhs, ao_rhs, strides, shape, nset, tab, ldtab,
        ))
    }

    pub fn try_aodmao2rho_loop_parallel<const BLKSIZE: usize>(
        rhos: &mut [f64], dms: &[f64], ao_lhs: &[f64], ao_rhs: &[f64], strides: [usize; 2],
        shape: [usize; 2], nset: usize, tab: &[bool], ldtab: usize,
    ) -> Result<(), Error> {
        let [stride_ao, stride_grid] = strides;
        let [nao, ngrid] = shape;
        status(unsafe {
            ffi::cfgmm_aodmao2rho_loop_parallel(
                rhos.as_mut_ptr(), rhos.len(), dms.as_ptr(), dms.len(), ao_lhs.as_ptr(),
                ao_lhs.len(), ao_rhs.as_ptr(), ao_rhs.len(), stride_ao, stride_grid, nao, ngrid,
                nset, tab_ptr(tab), tab.len(), ldtab, BLKSIZE,
            )
        })
    }
}

/// The f32 instantiation the reference's generic type allows
/// (src/structs.rs:3-13) but does not implement: f32 in and out, f64 inside,
/// one rounding at the end.
impl<const MC: usize, const KC: usize, const NC: usize, const MR: usize, const NR_LANE: usize, const LANE: usize>
    MatmulLoops<f32, MC, KC, NC, MR, NR_LANE, LANE>
{
    pub fn matmul_loop_parallel_mnk_pack_a(
        c: &mut [f32], a: &[f32], b: &[f32], m: usize, n: usize, k: usize, lda: usize,
        ldb: usize, ldc: usize, transa: bool, transb: bool,
    ) {
        or_panic(status(unsafe {
            ffi::cfgmm_matmul_f32(
                c.as_mut_ptr(), c.len(), a.as_ptr(), a.len(), b.as_ptr(), b.len(), m, n, k, lda,
                ldb, ldc, transa as u8, transb as u8, ffi::CFGMM_PREC_FP64,
            )
        }))
    }

    pub fn aodmao2rho_loop_parallel<const BLKSIZE: usize>(
        rhos: &mut [f32], dms: &[f32], ao_lhs: &[f32], ao_rhs: &[f32], strides: [usize; 2],
        shape: [usize; 2], nset: usize, tab: &[bool], ldtab: usize,
    ) {
        let [stride_ao, stride_grid] = strides;
        let [nao, ngrid] = shape;
        or_panic(status(unsafe {
            ffi::cfgmm_aodmao2rho_f32(
                rhos.as_mut_ptr(), rhos.len(), dms.as_ptr(), dms.len(), ao_lhs.as_ptr(),
                ao_lhs.len(), ao_rhs.as_ptr(), ao_rhs.len(), stride_ao, stride_grid, nao, ngrid,
                nset, tab_ptr(tab), tab.len(), ldtab, BLKSIZE, ffi::CFGMM_PREC_FP64,
            )
        }))
    }
}

/// The reference's `structs` module path.
pub mod structs {
    pub use crate::MatmulLoops;
}

/// The reference's `impl_matmul` module path.
pub mod impl_matmul {
    use super::*;

    /// src/impl_matmul.rs:234-248 (the reference's fixed Zen4 tuning).
    pub fn matmul_anyway_full(
        c: &mut [f64], a: &[f64], b: &[f64], m: usize, n: usize, k: usize, lda: usize,
        ldb: usize, ldc: usize, transa: bool, transb: bool,
    ) {
        or_panic(status(unsafe {
            ffi::cfgmm_matmul_anyway_full(
                c.as_mut_ptr(), c.len(), a.as_ptr(), a.len(), b.as_ptr(), b.len(), m, n, k, lda,
                ldb, ldc, transa as u8, transb as u8,
            )
        }))
    }

    /// The same product in an explicit arithmetic.
    pub fn matmul_ex(
        c: &mut [f64], a: &[f64], b: &[f64], m: usize, n: usize, k: usize, lda: usize,
        ldb: usize, ldc: usize, transa: bool, transb: bool, precision: Precision,
    ) -> Result<(), Error> {
        status(unsafe {
            ffi::cfgmm_matmul_ex(
                c.as_mut_ptr(), c.len(), a.as_ptr(), a.len(), b.as_ptr(), b.len(), m, n, k, lda,
                ldb, ldc, transa as u8, transb as u8, precision.code(),
            )
        })
    }
}

/// The reference's `impl_matmul_non0tab` module path.
pub mod impl_matmul_non0tab {
    use super::*;

    /// src/impl_matmul_non0tab.rs:308-326 (BLKSIZE 48).
    pub fn matmul_anyway_full_non0tab(
        c: &mut [f64], a: &[f64], b: &[f64], m: usize, n: usize, k: usize, lda: usize,
        ldb: usize, ldc: usize, transa: bool, transb: bool, tab: &[bool], ldtab: usize,
    ) {
        or_panic(status(unsafe {
            ffi::cfgmm_matmul_anyway_full_non0tab(
                c.as_mut_ptr(), c.len(), a.as_ptr(), a.len(), b.as_ptr(), b.len(), m, n, k, lda,
                ldb, ldc, transa as u8, transb as u8, tab_ptr(tab), tab.len(), ldtab,
            )
        }))
    }

    pub fn matmul_non0tab_ex(
        c: &mut [f64], a: &[f64], b: &[f64], m: usize, n: usize, k: usize, lda: usize,
        ldb: usize, ldc: usize, transa: bool, transb: bool, tab: &[bool], ldtab: usize,
        blksize: usize, precision: Precision,
    ) -> Result<(), Error> {
        status(unsafe {
            ffi::cfgmm_matmul_non0tab_ex(
                c.as_mut_ptr(), c.len(), a.as_ptr(), a.len(), b.as_ptr(), b.len(), m, n, k, lda,
                ldb, ldc, transa as u8, transb as u8, tab_ptr(tab), tab.len(), ldtab, blksize,
                precision.code(),
            )
        })
    }
}

/// The reference's `impl_aodmao2rho` module path.
pub mod impl_aodmao2rho {
    use super::*;

    /// src/impl_aodmao2rho.rs:247-261 (BLKSIZE 48).
    pub fn aodmao2rho_anyway(
        rhos: &mut [f64], dms: &[f64], ao_lhs: &[f64], ao_rhs: &[f64], strides: [usize; 2],
        shape: [usize; 2], nset: usize, tab: &[bool], ldtab: usize,
    ) {
        let [stride_ao, stride_grid] = strides;
        let [nao, ngrid] = shape;
        or_panic(status(unsafe {
            ffi::cfgmm_aodmao2rho_anyway(
                rhos.as_mut_ptr(), rhos.len(), dms.as_ptr(), dms.len(), ao_lhs.as_ptr(),
                ao_lhs.len(), ao_rhs.as_ptr(), ao_rhs.len(), stride_ao, stride_grid, nao, ngrid,
                nset, tab_ptr(tab), tab.len(), ldtab,
            )
        }))
    }

    /// The contraction in an explicit arithmetic, any BLKSIZE.
    pub fn aodmao2rho_ex(
        rhos: &mut [f64], dms: &[f64], ao_lhs: &[f64], ao_rhs: &[f64], strides: [usize; 2],
        shape: [usize; 2], nset: usize, tab: &[bool], ldtab: usize, blksize: usize,
        precision: Precision,
    ) -> Result<(), Error> {
        let [stride_ao, stride_grid] = strides;
        let [nao, ngrid] = shape;
        status(unsafe {
            ffi::cfgmm_aodmao2rho_ex(
                rhos.as_mut_ptr(), rhos.len(), dms.as_ptr(), dms.len(), ao_lhs.as_ptr(),
                ao_lhs.len(), ao_rhs.as_ptr(), ao_rhs.len(), stride_ao, stride_grid, nao, ngrid,
                nset, tab_ptr(tab), tab.len(), ldtab, blksize, precision.code(),
            )
        })
    }
}

pub use impl_aodmao2rho::aodmao2rho_anyway;
pub use impl_matmul::matmul_anyway_full;
pub use impl_matmul_non0tab::matmul_anyway_full_non0tab;

/// The library version, major * 10000 + minor * 100 + patch.
pub fn version() -> i32 {
    unsafe { ffi::cfgmm_version() }
}
