// Links libspectral_cuda.so (built by `python spectral_b200/build.py`, CUDA
// runtime linked statically into it).  SPECTRAL_CUDA_LIB_DIR names the
// directory that holds it; at run time the loader must find it too (rpath
// below, or LD_LIBRARY_PATH).
fn main() {
    println!("cargo:rerun-if-env-changed=SPECTRAL_CUDA_LIB_DIR");
    let dir = std::env::var("SPECTRAL_CUDA_LIB_DIR")
        .expect("set SPECTRAL_CUDA_LIB_DIR to the directory of libspectral_cuda.so");
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=spectral_cuda");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{dir}");
}
