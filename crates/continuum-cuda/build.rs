//! Links libcontinuum_cuda.so from CONTINUUM_CUDA_LIB_DIR (the directory
//! `python -m continuum_b200.build` writes it to: continuum_b200/lib).

fn main() {
    println!("cargo:rerun-if-env-changed=CONTINUUM_CUDA_LIB_DIR");
    let dir = std::env::var("CONTINUUM_CUDA_LIB_DIR")
        .expect("CONTINUUM_CUDA_LIB_DIR: the directory holding libcontinuum_cuda.so");
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=continuum_cuda");
}
