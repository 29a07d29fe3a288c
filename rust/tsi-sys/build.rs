// Links the static library libtsi.a (nvcc -lib, sm_100a) built by
// temporalsetinversion_b200/build.py, with the CUDA runtime it needs.
fn main() {
    let dir = std::env::var("TSI_LIB_DIR").unwrap_or_else(|_| "../../temporalsetinversion_b200/_lib".into());
    let cuda = std::env::var("CUDA_LIB_DIR").unwrap_or_else(|_| "/usr/local/cuda/lib64".into());
    println!("cargo:rustc-link-search=native={}", dir);
    println!("cargo:rustc-link-search=native={}", cuda);
    println!("cargo:rustc-link-lib=static=tsi");
    println!("cargo:rustc-link-lib=static=cudart_static");
    println!("cargo:rustc-link-lib=dylib=stdc++");
    println!("cargo:rustc-link-lib=dylib=rt");
    println!("cargo:rustc-link-lib=dylib=dl");
    println!("cargo:rustc-link-lib=dylib=pthread");
    println!("cargo:rerun-if-changed={}/libtsi.a", dir);
}
