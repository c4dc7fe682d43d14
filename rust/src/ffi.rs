//! Raw bindings of every entry point that `include/cfgmm.h` declares, in the
//! header's order.  Types follow the header one to one: `size_t` is `usize`,
//! `uint8_t` is `u8` (a Rust `bool` is passed as one byte 0/1; `&[bool]` as
//! `*const u8`), `int` is `c_int`, `cudaStream_t` / `cudaEvent_t` are
//! `*mut c_void`.  The header is the contract; the CPU test
//! `tests/test_rust_binding.py` checks names, argument counts and argument
//! widths here against it and against the symbols libcfgmm.so exports.
#![allow(non_camel_case_types)]

use core::ffi::{c_char, c_int, c_void};

pub const CFGMM_OK: c_int = 0;
pub const CFGMM_ERR_INVALID_ARGUMENT: c_int = -1;
pub const CFGMM_ERR_UNIMPLEMENTED: c_int = -2;
pub const CFGMM_ERR_CUDA: c_int = -3;
pub const CFGMM_ERR_NO_DEVICE: c_int = -4;
pub const CFGMM_ERR_OUT_OF_MEMORY: c_int = -5;
pub const CFGMM_ERR_TIMEOUT: c_int = -6;
pub const CFGMM_ERR_BUSY: c_int = -7;

pub const CFGMM_PREC_FP64: c_int = 0;
pub const CFGMM_PREC_OZAKI_INT8: c_int = 1;

pub const CFGMM_PLAN_NO_GRAPH: c_int = 1;
pub const CFGMM_PLAN_NO_TUNE: c_int = 2;

pub const CFGMM_NOALLOC_SCRATCH_BYTES: usize = 32 << 20;

/// One grid batch of a plan (`cfgmm_aodm_batch`), device pointers.
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct cfgmm_aodm_batch {
    pub rhos: *mut f64,
    pub ao_lhs: *const f64,
    pub ao_rhs: *const f64,
    pub tab: *const u8,
    pub stride_grid: usize,
    pub ngrid: usize,
    pub ldtab: usize,
    pub nset: usize,
}

/// Opaque plan handle.
#[repr(C)]
pub struct cfgmm_aodm_plan {
    _private: [u8; 0],
}

/// Opaque server handle.
#[repr(C)]
pub struct cfgmm_server {
    _private: [u8; 0],
}

/// Timings of one served request (`cfgmm_request_stats`).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct cfgmm_request_stats {
    pub queue_ms: f64,
    pub device_ms: f64,
    pub total_ms: f64,
    pub flops: f64,
}

extern "C" {
    pub fn cfgmm_status_string(status: c_int) -> *const c_char;
    pub fn cfgmm_last_error() -> *const c_char;
    pub fn cfgmm_version() -> c_int;

    // ---- 1. DGEMM --------------------------------------------------------
    pub fn cfgmm_matmul_loop_parallel_mnk_pack_a(
        c: *mut f64, c_len: usize, a: *const f64, a_len: usize, b: *const f64, b_len: usize,
        m: usize, n: usize, k: usize, lda: usize, ldb: usize, ldc: usize, transa: u8, transb: u8,
    ) -> c_int;
    pub fn cfgmm_matmul_anyway_full(
        c: *mut f64, c_len: usize, a: *const f64, a_len: usize, b: *const f64, b_len: usize,
        m: usize, n: usize, k: usize, lda: usize, ldb: usize, ldc: usize, transa: u8, transb: u8,
    ) -> c_int;
    pub fn cfgmm_matmul_loop_macro_mb(
        c: *mut f64, c_len: usize, a: *const f64, a_len: usize, b: *const f64, b_len: usize,
        m: usize, n: usize, k: usize, lda: usize, ldb: usize, ldc: usize, transa: u8, transb: u8,
    ) -> c_int;
    pub fn cfgmm_matmul_ex(
        c: *mut f64, c_len: usize, a: *const f64, a_len: usize, b: *const f64, b_len: usize,
        m: usize, n: usize, k: usize, lda: usize, ldb: usize, ldc: usize, transa: u8, transb: u8,
        precision: c_int,
    ) -> c_int;
    pub fn cfgmm_matmul_dev(
        c: *mut f64, a: *const f64, b: *const f64, m: usize, n: usize, k: usize, lda: usize,
        ldb: usize, ldc: usize, transa: u8, transb: u8, precision: c_int, stream: *mut c_void,
    ) -> c_int;
    pub fn cfgmm_matmul_anyway_full_non0tab(
        c: *mut f64, c_len: usize, a: *const f64, a_len: usize, b: *const f64, b_len: usize,
        m: usize, n: usize, k: usize, lda: usize, ldb: usize, ldc: usize, transa: u8, transb: u8,
        tab: *const u8, tab_len: usize, ldtab: usize,
    ) -> c_int;
    pub fn cfgmm_matmul_loop_parallel_mnk_pack_a_non0tab(
        c: *mut f64, c_len: usize, a: *const f64, a_len: usize, b: *const f64, b_len: usize,
        m: usize, n: usize, k: usize, lda: usize, ldb: usize, ldc: usize, transa: u8, transb: u8,
        tab: *const u8, tab_len: usize, ldtab: usize, blksize: usize,
    ) -> c_int;
    pub fn cfgmm_matmul_non0tab_ex(
        c: *mut f64, c_len: usize, a: *const f64, a_len: usize, b: *const f64, b_len: usize,
        m: usize, n: usize, k: usize, lda: usize, ldb: usize, ldc: usize, transa: u8, transb: u8,
        tab: *const u8, tab_len: usize, ldtab: usize, blksize: usize, precision: c_int,
    ) -> c_int;
    pub fn cfgmm_matmul_non0tab_dev(
        c: *mut f64, a: *const f64, b: *const f64, m: usize, n: usize, k: usize, lda: usize,
        ldb: usize, ldc: usize, transa: u8, transb: u8, tab: *const u8, ldtab: usize,
        blksize: usize, precision: c_int, stream: *mut c_void,
    ) -> c_int;
    pub fn cfgmm_matmul_dev_timed(
        c: *mut f64, a: *const f64, b: *const f64, m: usize, n: usize, k: usize, lda: usize,
        ldb: usize, ldc: usize, transa: u8, transb: u8, precision: c_int, stream: *mut c_void,
        events: *const *mut c_void, nevents: c_int,
    ) -> c_int;
    pub fn cfgmm_split_moduli(k: usize) -> c_int;
    pub fn cfgmm_device_check() -> c_int;
    pub fn cfgmm_test_arm_wait_timeout(precision: c_int, wait_ms: f64) -> c_int;

    // ---- 2. masked AO-DM-AO ---------------------------------------------
    pub fn cfgmm_aodmao2rho_loop_parallel(
        rhos: *mut f64, rhos_len: usize, dms: *const f64, dms_len: usize, ao_lhs: *const f64,
        ao_lhs_len: usize, ao_rhs: *const f64, ao_rhs_len: usize, stride_ao: usize,
        stride_grid: usize, nao: usize, ngrid: usize, nset: usize, tab: *const u8,
        tab_len: usize, ldtab: usize, blksize: usize,
    ) -> c_int;
    pub fn cfgmm_aodmao2rho_anyway(
        rhos: *mut f64, rhos_len: usize, dms: *const f64, dms_len: usize, ao_lhs: *const f64,
        ao_lhs_len: usize, ao_rhs: *const f64, ao_rhs_len: usize, stride_ao: usize,
        stride_grid: usize, nao: usize, ngrid: usize, nset: usize, tab: *const u8,
        tab_len: usize, ldtab: usize,
    ) -> c_int;
    pub fn cfgmm_aodmao2rho_ex(
        rhos: *mut f64, rhos_len: usize, dms: *const f64, dms_len: usize, ao_lhs: *const f64,
        ao_lhs_len: usize, ao_rhs: *const f64, ao_rhs_len: usize, stride_ao: usize,
        stride_grid: usize, nao: usize, ngrid: usize, nset: usize, tab: *const u8,
        tab_len: usize, ldtab: usize, blksize: usize, precision: c_int,
    ) -> c_int;
    pub fn cfgmm_aodmao2rho_dev(
        rhos: *mut f64, dms: *const f64, ao_lhs: *const f64, ao_rhs: *const f64,
        stride_ao: usize, stride_grid: usize, nao: usize, ngrid: usize, nset: usize,
        tab: *const u8, ldtab: usize, blksize: usize, precision: c_int, stream: *mut c_void,
    ) -> c_int;
    pub fn cfgmm_aodmao2rho_dev_noalloc(
        rhos: *mut f64, dms: *const f64, ao_lhs: *const f64, ao_rhs: *const f64,
        stride_ao: usize, stride_grid: usize, nao: usize, ngrid: usize, nset: usize,
        tab: *const u8, ldtab: usize, blksize: usize, stream: *mut c_void,
    ) -> c_int;
    pub fn cfgmm_aodm_fock(
        vs: *mut f64, vs_len: usize, ws: *const f64, ws_len: usize, ao_lhs: *const f64,
        ao_lhs_len: usize, ao_rhs: *const f64, ao_rhs_len: usize, stride_ao: usize,
        stride_grid: usize, nao: usize, ngrid: usize, nset: usize, tab: *const u8,
        tab_len: usize, ldtab: usize, blksize: usize,
    ) -> c_int;
    pub fn cfgmm_aodm_fock_dev(
        vs: *mut f64, ws: *const f64, ao_lhs: *const f64, ao_rhs: *const f64, stride_ao: usize,
        stride_grid: usize, nao: usize, ngrid: usize, nset: usize, tab: *const u8, ldtab: usize,
        blksize: usize, stream: *mut c_void,
    ) -> c_int;

    // ---- f32 forms -------------------------------------------------------
    pub fn cfgmm_matmul_f32(
        c: *mut f32, c_len: usize, a: *const f32, a_len: usize, b: *const f32, b_len: usize,
        m: usize, n: usize, k: usize, lda: usize, ldb: usize, ldc: usize, transa: u8, transb: u8,
        precision: c_int,
    ) -> c_int;
    pub fn cfgmm_matmul_f32_dev(
        c: *mut f32, a: *const f32, b: *const f32, m: usize, n: usize, k: usize, lda: usize,
        ldb: usize, ldc: usize, transa: u8, transb: u8, precision: c_int, stream: *mut c_void,
    ) -> c_int;
    pub fn cfgmm_aodmao2rho_f32(
        rhos: *mut f32, rhos_len: usize, dms: *const f32, dms_len: usize, ao_lhs: *const f32,
        ao_lhs_len: usize, ao_rhs: *const f32, ao_rhs_len: usize, stride_ao: usize,
        stride_grid: usize, nao: usize, ngrid: usize, nset: usize, tab: *const u8,
        tab_len: usize, ldtab: usize, blksize: usize, precision: c_int,
    ) -> c_int;
    pub fn cfgmm_aodmao2rho_f32_dev(
        rhos: *mut f32, dms: *const f32, ao_lhs: *const f32, ao_rhs: *const f32,
        stride_ao: usize, stride_grid: usize, nao: usize, ngrid: usize, nset: usize,
        tab: *const u8, ldtab: usize, blksize: usize, precision: c_int, stream: *mut c_void,
    ) -> c_int;

    // ---- batched plans ---------------------------------------------------
    pub fn cfgmm_aodm_plan_create(
        plan: *mut *mut cfgmm_aodm_plan, batches: *const cfgmm_aodm_batch, nbatch: usize,
        dms: *const f64, stride_ao: usize, nao: usize, nset_max: usize, blksize: usize,
        precision: c_int, flags: c_int, stream: *mut c_void,
    ) -> c_int;
    pub fn cfgmm_aodm_plan_run(plan: *mut cfgmm_aodm_plan, stream: *mut c_void) -> c_int;
    pub fn cfgmm_aodm_plan_info(plan: *const cfgmm_aodm_plan) -> *const c_char;
    pub fn cfgmm_aodm_plan_destroy(plan: *mut cfgmm_aodm_plan) -> c_int;

    // ---- AO evaluation on the device -------------------------------------
    pub fn cfgmm_eval_ao_dev(
        ao: *mut f64, stride_grid: usize, points: *const f64, ngrid: usize,
        shell_xyz: *const f64, shell_l: *const c_int, shell_alpha: *const f64,
        shell_norm: *const f64, shell_row: *const c_int, nshell: usize,
        shell_block_max: *mut f64, blksize: usize, stream: *mut c_void,
    ) -> c_int;
    pub fn cfgmm_mask_ao_dev(
        ao: *mut f64, stride_grid: usize, ngrid: usize, shell_l: *const c_int,
        shell_row: *const c_int, nshell: usize, shell_block_max: *const f64, threshold: f64,
        tab: *mut u8, ldtab: usize, blksize: usize, stream: *mut c_void,
    ) -> c_int;
    pub fn cfgmm_release_workspace() -> c_int;

    // ---- serving ---------------------------------------------------------
    pub fn cfgmm_server_create(
        server: *mut *mut cfgmm_server, hbm_budget: usize, nslots: c_int, precision: c_int,
        blksize: usize,
    ) -> c_int;
    pub fn cfgmm_server_destroy(server: *mut cfgmm_server) -> c_int;
    pub fn cfgmm_server_open(
        server: *mut cfgmm_server, ao_lhs: *const f64, ao_rhs: *const f64, tab: *const u8,
        nao: usize, ngrid: usize, ldtab: usize, nset_max: usize, on_device: c_int,
        molecule: *mut u64,
    ) -> c_int;
    pub fn cfgmm_server_open_shells(
        server: *mut cfgmm_server, points: *const f64, ngrid: usize, shell_xyz: *const f64,
        shell_l: *const c_int, shell_alpha: *const f64, shell_norm: *const f64, nshell: usize,
        density: f64, nset_max: usize, molecule: *mut u64,
    ) -> c_int;
    pub fn cfgmm_server_close(server: *mut cfgmm_server, molecule: u64) -> c_int;
    pub fn cfgmm_server_submit(
        server: *mut cfgmm_server, molecule: u64, dms: *const f64, nset: usize, rhos: *mut f64,
        ticket: *mut u64,
    ) -> c_int;
    pub fn cfgmm_server_submit_dev(
        server: *mut cfgmm_server, molecule: u64, dms: *const f64, nset: usize, rhos: *mut f64,
        stream: *mut c_void, ticket: *mut u64,
    ) -> c_int;
    pub fn cfgmm_server_wait(
        server: *mut cfgmm_server, ticket: u64, timeout_s: f64,
        stats: *mut cfgmm_request_stats,
    ) -> c_int;
    pub fn cfgmm_server_stats(server: *mut cfgmm_server) -> *const c_char;
}
