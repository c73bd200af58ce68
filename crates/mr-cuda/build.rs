// Links libmr_cuda.so.  MR_CUDA_LIB_DIR names the folder that holds it (the
// engine builds it in place at metal-route_b200/mrcuda/); the CUDA runtime is
// linked into the library itself, so nothing else is needed at link time.
fn main() {
    println!("cargo:rerun-if-env-changed=MR_CUDA_LIB_DIR");
    let dir = std::env::var("MR_CUDA_LIB_DIR").unwrap_or_else(|_| "../../metal-route_b200/mrcuda".into());
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=mr_cuda");
    // the tests and binaries find the library at run time without LD_LIBRARY_PATH
    println!("cargo:rustc-link-arg=-Wl,-rpath,{dir}");
}
