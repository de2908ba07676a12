// Links libwavefront_gpu.so.  Point WAVEFRONT_GPU_LIB_DIR at the directory
// that holds it (the library's own build writes wavefront_b200/lib/); the
// library links the CUDA runtime statically, so nothing else is needed.
fn main() {
    println!("cargo:rerun-if-env-changed=WAVEFRONT_GPU_LIB_DIR");
    if let Ok(dir) = std::env::var("WAVEFRONT_GPU_LIB_DIR") {
        println!("cargo:rustc-link-search=native={dir}");
    }
    println!("cargo:rustc-link-lib=dylib=wavefront_gpu");
}
