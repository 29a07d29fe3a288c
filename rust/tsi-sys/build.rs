// Links libtsi.so built by temporalsetinversion_b200/build.py.
fn main() {
    let dir = std::env::var("TSI_LIB_DIR").unwrap_or_else(|_| "../../temporalsetinversion_b200/_lib".into());
    println!("cargo:rustc-link-search=native={}", dir);
    println!("cargo:rustc-link-lib=dylib=tsi");
}
