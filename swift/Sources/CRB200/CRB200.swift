// CRB200.swift — a thin Swift layer over the B200 compute rasteriser's C ABI
// (include/cr/cr.h), keeping the method names of the reference's Swift API so
// that a renderer written against SatinComputeRasteriser moves over with few
// changes:
//   ComputeRasteriser           update / encode / pickPointIndex
//                               (Sources/SatinComputeRasteriser/ComputeRasteriser.swift:201-296, 609-670)
//   ComputeRasteriserPointCloud addBatches / removeBatches / commitBatchUpdates / updateFiles
//                               (Sources/SatinComputeRasteriser/ComputeRasteriserPointCloud.swift:410-515)
// Metal objects become the library's handles: the output is read back as
// RGBA8 bytes instead of being a texture, and the camera is the pair of
// column-major view / projection matrices the reference takes from Satin.
//
// Unverified: no Swift toolchain was available where this was written; the
// Python mirror (satin-computerasteriser_b200/__init__.py) is the tested host
// layer over the same calls.
import CCRB200

public enum ComputeRasteriserMode: Int32 {
    case highQualityAverage = 0
    case nearestPoint = 1
}

/// A failed library call: the cr_status and the library's detail text.
public struct CRError: Error, CustomStringConvertible {
    public let status: cr_status
    public let detail: String
    public var description: String {
        String(cString: cr_status_string(status)) + ": " + detail
    }
}

@inline(__always)
func check(_ status: cr_status) throws {
    if status != CR_OK {
        throw CRError(status: status, detail: String(cString: cr_last_error_detail()))
    }
}

/// Column-major 4x4 float matrix, as the ABI takes it.
public typealias CRMatrix = [Float]  // 16 values

/// The camera as the reference's processors receive it (viewMatrix, projectionMatrix).
public struct CRCamera {
    public var view: CRMatrix
    public var projection: CRMatrix
    public init(view: CRMatrix, projection: CRMatrix) {
        precondition(view.count == 16 && projection.count == 16)
        self.view = view
        self.projection = projection
    }
    var c: cr_camera {
        var cam = cr_camera()
        withUnsafeMutableBytes(of: &cam.view) { dst in view.withUnsafeBytes { dst.copyMemory(from: $0) } }
        withUnsafeMutableBytes(of: &cam.projection) { dst in
            projection.withUnsafeBytes { dst.copyMemory(from: $0) }
        }
        return cam
    }
}

/// a * b for column-major matrices with the library's operation order.
func multiply(_ a: CRMatrix, _ b: CRMatrix) -> CRMatrix {
    var out = CRMatrix(repeating: 0, count: 16)
    for c in 0..<4 {
        for r in 0..<4 {
            let s0 = a[r] * b[4 * c] + a[4 + r] * b[4 * c + 1]
            out[4 * c + r] = (s0 + a[8 + r] * b[4 * c + 2]) + a[12 + r] * b[4 * c + 3]
        }
    }
    return out
}

/// One CUDA device and its stream (the reference's Satin Context).
public final class CRContext {
    let handle: OpaquePointer
    public init(device: Int32 = 0) throws {
        var h: OpaquePointer?
        try check(cr_context_create(device, &h))
        handle = h!
    }
    deinit { cr_context_destroy(handle) }
    public func synchronize() throws { try check(cr_context_synchronize(handle)) }
}

/// ComputeRasteriserCapacity (ComputeRasteriserPointCloud.swift:23-40).
public struct ComputeRasteriserCapacity {
    public var maxResidentBatches: Int
    public var pointsPerBatch: Int
    public init(maxResidentBatches: Int, pointsPerBatch: Int = Int(CR_DEFAULT_POINTS_PER_BATCH)) {
        self.maxResidentBatches = maxResidentBatches
        self.pointsPerBatch = pointsPerBatch
    }
}

/// The slot pool of one cloud (ComputeRasteriserPointCloud).
public final class ComputeRasteriserPointCloud {
    let handle: OpaquePointer
    public let capacity: ComputeRasteriserCapacity
    public var worldMatrix: CRMatrix = [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1]

    public init(context: CRContext, capacity: ComputeRasteriserCapacity,
                files: [cr_raster_file]? = nil) throws {
        self.capacity = capacity
        var h: OpaquePointer?
        let cap = cr_capacity(maxResidentBatches: UInt32(capacity.maxResidentBatches),
                              pointsPerBatch: UInt32(capacity.pointsPerBatch))
        if let files {
            try files.withUnsafeBufferPointer {
                try check(cr_cloud_create(context.handle, cap, $0.baseAddress, UInt32($0.count), &h))
            }
        } else {
            try check(cr_cloud_create(context.handle, cap, nil, 0, &h))
        }
        handle = h!
    }
    deinit { cr_cloud_destroy(handle) }

    /// addBatches(positionsXYZLow:positionsXYZMed:positionsXYZHigh:colors:levels:batches:commit:);
    /// returns the slot of each batch.
    @discardableResult
    public func addBatches(positionsXYZLow: [UInt32], positionsXYZMed: [UInt32],
                           positionsXYZHigh: [UInt32], colors: [UInt32], levels: [UInt8],
                           batches: [cr_raster_batch], commit: Bool = true) throws -> [Int] {
        var slots = [Int32](repeating: -1, count: batches.count)
        let n = UInt64(colors.count)
        try positionsXYZLow.withUnsafeBufferPointer { lo in
            try positionsXYZMed.withUnsafeBufferPointer { me in
                try positionsXYZHigh.withUnsafeBufferPointer { hi in
                    try colors.withUnsafeBufferPointer { co in
                        try levels.withUnsafeBufferPointer { lv in
                            try batches.withUnsafeBufferPointer { b in
                                try check(cr_cloud_add_batches(
                                    handle, lo.baseAddress, me.baseAddress, hi.baseAddress,
                                    co.baseAddress, lv.baseAddress, n, b.baseAddress,
                                    UInt32(b.count), commit ? 1 : 0, &slots))
                            }
                        }
                    }
                }
            }
        }
        return slots.map { Int($0) }
    }

    /// removeBatches(slots:commit:).
    public func removeBatches(slots: [Int], commit: Bool = true) throws {
        let s = slots.map { Int32($0) }
        try s.withUnsafeBufferPointer {
            try check(cr_cloud_remove_batches(handle, $0.baseAddress, UInt32($0.count), commit ? 1 : 0))
        }
    }

    /// commitBatchUpdates().
    public func commitBatchUpdates() throws { try check(cr_cloud_commit(handle)) }

    /// updateFiles(viewProjection:modelMatrix:frustumTransform:prevViewProjection:).
    public func updateFiles(viewProjection: CRMatrix, modelMatrix: CRMatrix,
                            frustumTransform: CRMatrix? = nil,
                            prevViewProjection: CRMatrix? = nil) throws {
        let fr = frustumTransform ?? []
        let pv = prevViewProjection ?? []
        try viewProjection.withUnsafeBufferPointer { vp in
            try modelMatrix.withUnsafeBufferPointer { m in
                try fr.withUnsafeBufferPointer { f in
                    try pv.withUnsafeBufferPointer { p in
                        try check(cr_cloud_update_files(
                            handle, vp.baseAddress, m.baseAddress,
                            frustumTransform == nil ? nil : f.baseAddress,
                            prevViewProjection == nil ? nil : p.baseAddress))
                    }
                }
            }
        }
    }

    public var residentBatchCount: Int {
        var info = cr_cloud_info()
        cr_cloud_info_get(handle, &info)
        return Int(info.residentBatchCount)
    }
}

/// The per-frame render API (ComputeRasteriser).
public final class ComputeRasteriser {
    let context: CRContext
    public var configuration: cr_config
    public private(set) var pointClouds: [ComputeRasteriserPointCloud] = []
    var frame: OpaquePointer?
    var width = 0, height = 0
    var camera: CRCamera?

    public init(context: CRContext) throws {
        self.context = context
        var cfg = cr_config()
        try check(cr_config_default(&cfg))
        configuration = cfg
    }
    deinit { if let frame { cr_frame_destroy(frame) } }

    @discardableResult
    public func addPointCloud(_ cloud: ComputeRasteriserPointCloud) -> ComputeRasteriserPointCloud {
        pointClouds.append(cloud)
        return cloud
    }

    public func removePointCloud(_ cloud: ComputeRasteriserPointCloud) {
        pointClouds.removeAll { $0 === cloud }
    }

    /// resize(size:) — the viewport's buffers.
    public func resize(width: Int, height: Int) throws {
        guard width > 0, height > 0, width != self.width || height != self.height else { return }
        if let frame { cr_frame_destroy(frame) }
        var f: OpaquePointer?
        try check(cr_frame_create(context.handle, Int32(width), Int32(height), &f))
        frame = f
        self.width = width
        self.height = height
    }

    /// update(renderContext:camera:viewport:index:): sets the camera and
    /// refreshes every cloud's file table (viewProjection * world).
    public func update(camera: CRCamera, viewport: (width: Int, height: Int)? = nil) throws {
        if let viewport { try resize(width: viewport.width, height: viewport.height) }
        self.camera = camera
        let vp = multiply(camera.projection, camera.view)
        for cloud in pointClouds {
            try cloud.updateFiles(viewProjection: vp, modelMatrix: cloud.worldMatrix)
        }
    }

    /// encode(_:): enqueues the frame (HQS or nearest point, then hole fill).
    public func encode() throws {
        guard let frame, let camera else { return }
        var cfg = configuration
        var cam = camera.c
        let handles: [OpaquePointer?] = pointClouds.map { $0.handle }
        try handles.withUnsafeBufferPointer {
            try check(cr_render(context.handle, frame, $0.baseAddress, UInt32($0.count), &cfg, &cam))
        }
    }

    /// The frame's image as RGBA8 bytes (row 0 at the top); waits for the frame.
    public func outputRGBA8() throws -> [UInt8] {
        guard let frame else { return [] }
        var out = [UInt8](repeating: 0, count: width * height * 4)
        try out.withUnsafeMutableBufferPointer { try check(cr_frame_read_rgba8(frame, $0.baseAddress)) }
        return out
    }

    /// Enqueues the read-back of the frame's image into `out` (w*h*4 bytes,
    /// page-locked memory keeps the copy asynchronous) and returns at once;
    /// the copy overlaps the next encode() up to its resolve.  The caller
    /// keeps `out` alive until waitOutput covers this read-back.
    public func outputRGBA8Async(into out: UnsafeMutablePointer<UInt8>) throws {
        guard let frame else { return }
        try check(cr_frame_read_rgba8_async(frame, out))
    }

    /// Waits for the read-backs enqueued by outputRGBA8Async: all of them
    /// (keep 0), or all but the `keep` (at most 3) most recent.
    public func waitOutput(keep: Int = 0) throws {
        guard let frame else { return }
        try check(cr_frame_read_wait_keep(frame, Int32(keep)))
    }

    /// pickPointIndex(atNDC:in:camera:searchRadius:): the global packed point
    /// index under ndc (y up), or nil.  Blocks until the GPU has finished.
    public func pickPointIndex(atNDC ndc: (Float, Float), in cloud: ComputeRasteriserPointCloud,
                               camera: CRCamera, searchRadius: Int = 10) throws -> UInt32? {
        guard let frame else { return nil }
        var cfg = configuration
        var cam = camera.c
        let p: [Float] = [ndc.0, ndc.1]
        var index: UInt32 = 0
        var found: Int32 = 0
        try p.withUnsafeBufferPointer {
            try check(cr_pick(context.handle, frame, cloud.handle, $0.baseAddress, &cfg, &cam,
                              Int32(searchRadius), &index, &found))
        }
        return found != 0 ? index : nil
    }
}
