// Links libnatsel_gpu.so. Build it first (python -c "import natsel_b200._build as b; b.build()",
// which writes natsel_b200/libnatsel_gpu.so for sm_100a); NATSEL_GPU_LIB_DIR overrides where it
// is looked for.
use std::env;
use std::path::PathBuf;

fn main() {
    let dir = env::var("NATSEL_GPU_LIB_DIR").map(PathBuf::from).unwrap_or_else(|_| {
        PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap()).join("..").join("natsel_b200")
    });
    println!("cargo:rerun-if-env-changed=NATSEL_GPU_LIB_DIR");
    println!("cargo:rerun-if-changed=../include/natsel_gpu.h");
    println!("cargo:rustc-link-search=native={}", dir.display());
    println!("cargo:rustc-link-lib=dylib=natsel_gpu");
}
