//! Builds libprg_b200.so from the CUDA sources with nvcc for sm_100a and
//! tells cargo to link it.  The flags are those of rust-igraph_b200/build.py.
//! Environment: NVCC (default "nvcc"), PRG_B200_CSRC (default ../csrc).
use std::env;
use std::path::{Path, PathBuf};
use std::process::Command;

fn nvcc() -> String {
    env::var("NVCC").unwrap_or_else(|_| "nvcc".to_string())
}

fn main() {
    let manifest = PathBuf::from(env::var("CARGO_MANIFEST_DIR").expect("CARGO_MANIFEST_DIR"));
    let csrc = env::var("PRG_B200_CSRC").map(PathBuf::from).unwrap_or_else(|_| manifest.join("../csrc"));
    let include = manifest.join("../../include");
    let out = PathBuf::from(env::var("OUT_DIR").expect("OUT_DIR"));
    let arch = ["-gencode", "arch=compute_100a,code=sm_100a"];
    let flags = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"];

    let mut sources: Vec<PathBuf> = std::fs::read_dir(&csrc)
        .unwrap_or_else(|e| panic!("reading {}: {e}", csrc.display()))
        .filter_map(|d| d.ok().map(|d| d.path()))
        .collect();
    sources.sort();
    let mut objects = Vec::new();
    for src in &sources {
        let ext = src.extension().and_then(|e| e.to_str()).unwrap_or("");
        if ext == "cuh" || ext == "h" {
            println!("cargo:rerun-if-changed={}", src.display());
            continue;
        }
        if ext != "cu" {
            continue;
        }
        println!("cargo:rerun-if-changed={}", src.display());
        let stem = src.file_stem().and_then(|s| s.to_str()).expect("source name");
        let obj = out.join(format!("{stem}.o"));
        let status = Command::new(nvcc())
            .args(arch)
            .args(flags)
            .arg("-I")
            .arg(&include)
            .arg("-I")
            .arg(&csrc)
            .arg("-c")
            .arg(src)
            .arg("-o")
            .arg(&obj)
            .status()
            .expect("running nvcc");
        assert!(status.success(), "nvcc failed on {}", src.display());
        objects.push(obj);
    }
    println!("cargo:rerun-if-changed={}", include.join("prg_b200.h").display());
    println!("cargo:rerun-if-env-changed=NVCC");
    println!("cargo:rerun-if-env-changed=PRG_B200_CSRC");

    let lib = out.join("libprg_b200.so");
    let status = Command::new(nvcc())
        .args(arch)
        .arg("-shared")
        .arg("-o")
        .arg(&lib)
        .args(&objects)
        .arg("-lcudart")
        .status()
        .expect("running nvcc to link");
    assert!(status.success(), "linking {} failed", lib.display());

    println!("cargo:rustc-link-search=native={}", out.display());
    println!("cargo:rustc-link-lib=dylib=prg_b200");
    // let binaries find the library next to the build output
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", Path::new(&out).display());
}
