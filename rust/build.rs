//! Builds libcfgmm.so with nvcc (sm_100a) through the repository's build
//! script and links it.  The library carries the CUDA runtime statically, so
//! only the NVIDIA driver is needed at run time.
//!
//! Environment:
//!   CFGMM_ROOT    checkout of this repository (default: the parent of this crate)
//!   CFGMM_PYTHON  Python interpreter that runs the build script (default: python3)
//!   CFGMM_NO_BUILD=1  link an already-built library without running nvcc
use std::env;
use std::path::PathBuf;
use std::process::Command;

fn main() {
    let manifest = PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap());
    let root = env::var("CFGMM_ROOT")
        .map(PathBuf::from)
        .unwrap_or_else(|_| manifest.parent().expect("crate inside the checkout").to_path_buf());
    let pkg = root.join("cfgable-matmul_b200");
    if env::var("CFGMM_NO_BUILD").map(|v| v != "1").unwrap_or(true) {
        let python = env::var("CFGMM_PYTHON").unwrap_or_else(|_| "python3".to_string());
        let status = Command::new(python)
            .arg(pkg.join("build.py"))
            .status()
            .expect("running cfgable-matmul_b200/build.py (needs nvcc)");
        assert!(status.success(), "building libcfgmm.so failed");
    }
    println!("cargo:rustc-link-search=native={}", pkg.display());
    println!("cargo:rustc-link-lib=dylib=cfgmm");
    // find the library next to the checkout at run time without LD_LIBRARY_PATH
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", pkg.display());
    println!("cargo:rerun-if-changed={}", pkg.join("csrc").display());
    println!("cargo:rerun-if-changed={}", root.join("include").join("cfgmm.h").display());
    println!("cargo:rerun-if-env-changed=CFGMM_ROOT");
    println!("cargo:rerun-if-env-changed=CFGMM_NO_BUILD");
}
