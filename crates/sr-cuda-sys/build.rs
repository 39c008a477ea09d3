//! Builds libsrcuda from the CUDA sources beside this crate (nvcc, sm_100a) and links it statically.
//!
//! Environment:
//!   NVCC              the nvcc to run (default: $CUDA_HOME/bin/nvcc, then /usr/local/cuda/bin/nvcc)
//!   CUDA_HOME         the CUDA toolkit (default /usr/local/cuda): its lib64 holds libcudart
//!   SR_CUDA_LIB_DIR   set to link a prebuilt libsrcuda.so from that directory instead of compiling
use std::env;
use std::path::{Path, PathBuf};
use std::process::Command;

const SOURCES: &[&str] = &[
    "ctx.cu", "box.cu", "hydro.cu",
    "hydro_ref.cu", "grav.cu", "grav_static.cu", "heat.cu", "mg.cu", "batch.cu", "learned.cu",
];

fn main() {
    let cuda = env::var("CUDA_HOME").unwrap_or_else(|_| "/usr/local/cuda".to_string());
    println!("cargo:rerun-if-env-changed=SR_CUDA_LIB_DIR");
    println!("cargo:rerun-if-env-changed=NVCC");
    println!("cargo:rerun-if-env-changed=CUDA_HOME");
    if let Ok(dir) = env::var("SR_CUDA_LIB_DIR") {
        println!("cargo:rustc-link-search=native={dir}");
        println!("cargo:rustc-link-lib=dylib=srcuda");
        return;
    }
    let manifest = PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap());
    let root = manifest.join("../..").canonicalize().expect("the repository root above crates/");
    let csrc = root.join("sandbox_reactions_b200/csrc");
    let include = root.join("include");
    let out = PathBuf::from(env::var("OUT_DIR").unwrap());
    let nvcc = env::var("NVCC").unwrap_or_else(|_| format!("{cuda}/bin/nvcc"));

    let mut objects = Vec::new();
    for src in SOURCES {
        let path = csrc.join(src);
        println!("cargo:rerun-if-changed={}", path.display());
        let obj = out.join(src.replace(".cu", ".o"));
        run(Command::new(&nvcc)
            .args(["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-lineinfo"])
            .args(["-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"])
            .arg("-I").arg(&include)
            .arg("-c").arg(&path)
            .arg("-o").arg(&obj));
        objects.push(obj);
    }
    for entry in std::fs::read_dir(&csrc).unwrap() {
        let p = entry.unwrap().path();
        if p.extension().map_or(false, |e| e == "cuh") {
            println!("cargo:rerun-if-changed={}", p.display());
        }
    }
    println!("cargo:rerun-if-changed={}", include.join("sr_cuda.h").display());
    // device code is linked once into the archive (relocatable device code is not used)
    let lib = out.join("libsrcuda.a");
    let _ = std::fs::remove_file(&lib);
    run(Command::new("ar").arg("crs").arg(&lib).args(&objects));
    println!("cargo:rustc-link-search=native={}", out.display());
    println!("cargo:rustc-link-lib=static=srcuda");
    println!("cargo:rustc-link-search=native={}", Path::new(&cuda).join("lib64").display());
    println!("cargo:rustc-link-lib=dylib=cudart");
    println!("cargo:rustc-link-lib=dylib=stdc++");
}

fn run(cmd: &mut Command) {
    let status = cmd.status().unwrap_or_else(|e| panic!("could not run {cmd:?}: {e}"));
    assert!(status.success(), "{cmd:?} failed with {status}");
}
