// Links libgalaxy_b200.so. GALAXY_B200_LIB_DIR points at the directory holding it
// (default: the package directory next to this crate, where __graft_entry__.build() puts it).
fn main() {
    let dir = std::env::var("GALAXY_B200_LIB_DIR").unwrap_or_else(|_| {
        let here = std::path::PathBuf::from(std::env::var("CARGO_MANIFEST_DIR").unwrap());
        here.join("../..").canonicalize().unwrap().display().to_string()
    });
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=galaxy_b200");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{dir}");
    println!("cargo:rerun-if-env-changed=GALAXY_B200_LIB_DIR");
}
