// swift-tools-version:5.9
// Swift binding of the B200 compute rasteriser's C ABI (include/cr/cr.h).
// Unverified: no Swift toolchain was available where this was written.
// Build the library first (python satin-computerasteriser_b200/build.py) and
// pass its directory to the linker, e.g.
//   swift build -Xlinker -L../satin-computerasteriser_b200/_lib
import PackageDescription

let package = Package(
    name: "CRB200",
    products: [.library(name: "CRB200", targets: ["CRB200"])],
    targets: [
        .systemLibrary(name: "CCRB200", path: "Sources/CCRB200"),
        .target(name: "CRB200", dependencies: ["CCRB200"], path: "Sources/CRB200"),
    ]
)
