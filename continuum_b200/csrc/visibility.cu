// The plain visibility kernel: one warp walks a packet of up to 32 cones
// (neighbouring points toward one light) through the scene hierarchy
// together; the lanes share the rasterization of every leaf the packet
// visits, and each lane integrates its own cone.
//
// What the reference does per invocation (mask_cones.wgsl `main` :1513-1520
// -> hit_irradiance_rect :2125 -> cone_irradiance_rect :1286) is done here
// per cone, with the packet walk of the reference's PACKETS mode
// (packet_any, :666-711) built from warp votes:
//  * the traversal stack is warp-uniform and lives in registers spread over
//    the lanes (entry i in lane i % 32), so a push is one predicated move and
//    a pop one shuffle — no shared or local memory;
//  * each lane keeps a bit per stack entry saying whether its own walk needs
//    that entry (need_get/need_put, :694-711);
//  * node and triangle records are loaded by every lane from the same
//    address, which the load unit serves as one broadcast transaction;
//  * at a triangle-hierarchy leaf, the (triangle, cone) pairs of every cone
//    that descends into it are dealt out over all 32 lanes, which cull and
//    rasterize them into the owning cone's accumulator — cones whose
//    triangles take the long clip path no longer hold 31 lanes idle.
// Results depend on the walk order only through the walk caps: the packet
// takes the child order most of its descending lanes prefer; a lane whose own
// nearest-first order differs somewhere on its walk, and whose walk then
// stopped early (capped, or every bin full), is listed and walked again
// alone by a second launch, so every cone's result is the one its own walk
// gives (the reference's walk without packets, as its view-cache bakes run).
#include "visibility_kernel.cuh"

namespace cc {

// ---- host-side launchers --------------------------------------------------------

cudaError_t upload_disk_table(const float* table64) {
  cudaError_t e = cudaMemcpyToSymbol(c_disk, table64, kBins * sizeof(float));
  if (e == cudaSuccess) e = upload_disk_table_split(table64);  // the integrating unit's copy
  if (e != cudaSuccess) return e;
  return upload_disk_table_splat(table64);  // the prefiltering unit's copy
}

// The exact cones' plain pass (packet or solo) of the variant the flags pick;
// prefiltering cones' passes are compiled in visibility_splat.cu.
template <bool kWide>
static cudaError_t exact_pass(bool count, bool inst, bool sky, const DevScene& s, const DevQuery& q, const DevOut& o,
                              const uint32_t* list, const uint32_t* list_count, uint32_t pw, uint32_t blocks,
                              cudaStream_t stream) {
  return sky ? plain_pass<kWide, true, false>(count, inst, s, q, o, list, list_count, pw, blocks, stream)
             : plain_pass<kWide, false, false>(count, inst, s, q, o, list, list_count, pw, blocks, stream);
}

// The split plain path (exact light cones): per chunk of at most `chunk`
// slots, the cones set up, walked (the packet pass, then the solo pass over
// the slots it listed) and integrated. The marks: after the first chunk's
// setup, after the last chunk's packet pass, after the last integration (a
// call of one chunk: its packet pass, then its solo pass and integration).
static cudaError_t split_visibility(const DevScene& s, const DevQuery& q0, const DevOut& o, uint32_t pw, bool count,
                                    bool inst, uint64_t chunk, int sm_count, cudaStream_t stream,
                                    const cudaEvent_t* marks, cudaEvent_t walked) {
  if (!q0.records || !o.cov_out || chunk == 0) return cudaErrorInvalidValue;
  const uint64_t ncones = q0.npoints * (uint64_t)q0.nlights;
  cudaError_t e = cudaSuccess;
  for (uint64_t base = 0; base < ncones; base += chunk) {
    const uint64_t n = ncones - base < chunk ? ncones - base : chunk;
    DevQuery q = q0;
    q.slot_base = base;
    q.slot_count = n;
    if (base > 0) {
      // Each chunk's passes count from zero again; the error word carries on.
      e = cudaMemsetAsync(o.redo_count, 0, sizeof(uint32_t), stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(o.next_packet, 0, sizeof(uint32_t), stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(o.next_solo, 0, sizeof(uint32_t), stream);
      if (e != cudaSuccess) return e;
    }
    e = launch_cone_setup(q, base, n, const_cast<ConeRecord*>(q.records), stream);
    if (e != cudaSuccess) return e;
    if (marks && base == 0) cudaEventRecord(marks[0], stream);
    const uint64_t packets = (n + pw - 1) / pw;
    const uint64_t want = (packets + kWarpsPerBlock - 1) / kWarpsPerBlock;
    const uint64_t cap = (uint64_t)sm_count * kBlocksPerSm;
    const uint32_t blocks = (uint32_t)(want < cap ? want : cap);
    e = plain_pass<false, false, false>(count, inst, s, q, o, nullptr, nullptr, pw, blocks, stream);
    if (e != cudaSuccess) return e;
    if (marks && base + chunk >= ncones) cudaEventRecord(marks[1], stream);
    if (o.redo_list) {
      e = plain_pass<true, false, false>(count, inst, s, q, o, o.redo_list, o.redo_count, 1,
                                         (uint32_t)sm_count * kSoloBlocksPerSm, stream);
      if (e != cudaSuccess) return e;
    }
    if (walked && base + chunk >= ncones) {
      e = cudaEventRecord(walked, stream);
      if (e != cudaSuccess) return e;
    }
    e = launch_integrate(q, o, base, n, q.records, stream);
    if (e != cudaSuccess) return e;
  }
  if (marks) cudaEventRecord(marks[2], stream);
  return e;
}

cudaError_t launch_visibility(const DevScene& s, const DevQuery& q, const DevOut& o, uint32_t pw, bool count,
                              uint64_t chunk, int sm_count, cudaStream_t stream, const cudaEvent_t* marks,
                              cudaEvent_t walked) {
  if (pw < 1) pw = 1;
  if (pw > 32) pw = 32;
  const uint64_t ncones = q.npoints * (uint64_t)q.nlights;
  if (ncones == 0) {
    if (marks) {
      cudaEventRecord(marks[0], stream);
      cudaEventRecord(marks[1], stream);
      cudaEventRecord(marks[2], stream);
    }
    return cudaSuccess;
  }
  const bool inst = s.xforms != nullptr;
  const bool sky = (q.sky & kSkyCones) != 0u;
  const bool splat = q.prefilter > 0.0f;
  if (!sky && !splat) return split_visibility(s, q, o, pw, count, inst, chunk, sm_count, stream, marks, walked);
  if (marks) cudaEventRecord(marks[0], stream);
  const uint64_t packets = (ncones + pw - 1) / pw;
  const uint64_t want = (packets + kWarpsPerBlock - 1) / kWarpsPerBlock;
  // One resident wave: warps take packets from the shared counter; the
  // blocks per SM follow where the variant keeps its coverages.
  const uint64_t cap = (uint64_t)sm_count * resident_blocks_for(false, sky, splat);
  const uint32_t blocks = (uint32_t)(want < cap ? want : cap);
  // The packet pass with 32-bit accumulator cells, the solo pass with 64-bit.
  auto packets_pass = [&](uint32_t p, uint32_t nb) {
    return splat ? launch_splat_pass(false, count, inst, sky, s, q, o, nullptr, nullptr, p, nb, stream)
                 : exact_pass<false>(count, inst, sky, s, q, o, nullptr, nullptr, p, nb, stream);
  };
  auto solo_pass = [&](uint32_t nb) {
    return splat ? launch_splat_pass(true, count, inst, sky, s, q, o, o.redo_list, o.redo_count, 1, nb, stream)
                 : exact_pass<true>(count, inst, sky, s, q, o, o.redo_list, o.redo_count, 1, nb, stream);
  };
  cudaError_t e = packets_pass(pw, blocks);
  if (marks) cudaEventRecord(marks[1], stream);
  if (e != cudaSuccess) return e;
  if (o.redo_list) {
    // The listed cones, each walked alone (one cone per warp; the warp still
    // shares its leaves' triangles).
    e = solo_pass((uint32_t)sm_count * resident_blocks_for(true, sky, splat));
  }
  if (marks) cudaEventRecord(marks[2], stream);
  return e;
}

cudaError_t launch_batch(const BatchLaunch& b0, const DevOut& o, const BatchChunk* chunks, size_t nchunks, bool count,
                         int sm_count, int blocks_per_sm, cudaStream_t stream) {
  if (b0.njobs == 0 || b0.packets == 0) return cudaSuccess;
  if (!b0.records || !o.cov_out) return cudaErrorInvalidValue;
  if (blocks_per_sm < 1) blocks_per_sm = 1;
  if (blocks_per_sm > kBlocksPerSm) blocks_per_sm = kBlocksPerSm;
  const DevScene s{};
  const DevQuery q{};
  cudaError_t e = cudaSuccess;
  for (size_t k = 0; k < nchunks; ++k) {
    BatchLaunch b = b0;
    b.packet_base = chunks[k].packet_base;
    b.packet_count = chunks[k].packet_count;
    b.cone_base = chunks[k].cone_base;
    b.cone_count = chunks[k].cone_count;
    if (k > 0) {
      // Each chunk's passes count from zero again; the error word carries on.
      e = cudaMemsetAsync(o.redo_count, 0, sizeof(uint32_t), stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(o.next_packet, 0, sizeof(uint32_t), stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(o.next_solo, 0, sizeof(uint32_t), stream);
      if (e != cudaSuccess) return e;
    }
    e = launch_batch_setup(b, stream);
    if (e != cudaSuccess) return e;
    const uint64_t want = (b.packet_count + kWarpsPerBlock - 1) / kWarpsPerBlock;
    const uint64_t cap = (uint64_t)sm_count * blocks_per_sm;
    const uint32_t blocks = (uint32_t)(want < cap ? want : cap);
    // Batches with an instanced scene take the instanced variant, which
    // walks world-space scenes too.
    if (b.inst) {
      e = count ? launch_one<true, true, true, false>(s, q, o, b, nullptr, nullptr, b.pw, blocks, stream)
                : launch_one<false, true, true, false>(s, q, o, b, nullptr, nullptr, b.pw, blocks, stream);
    } else {
      e = count ? launch_one<true, true, false, false>(s, q, o, b, nullptr, nullptr, b.pw, blocks, stream)
                : launch_one<false, true, false, false>(s, q, o, b, nullptr, nullptr, b.pw, blocks, stream);
    }
    if (e != cudaSuccess) return e;
    if (o.redo_list) {
      const uint32_t solo_blocks = (uint32_t)sm_count * kSoloBlocksPerSm;
      if (b.inst) {
        e = count ? launch_one<true, true, true, true>(s, q, o, b, o.redo_list, o.redo_count, 1, solo_blocks, stream)
                  : launch_one<false, true, true, true>(s, q, o, b, o.redo_list, o.redo_count, 1, solo_blocks, stream);
      } else {
        e = count ? launch_one<true, true, false, true>(s, q, o, b, o.redo_list, o.redo_count, 1, solo_blocks, stream)
                  : launch_one<false, true, false, true>(s, q, o, b, o.redo_list, o.redo_count, 1, solo_blocks, stream);
      }
      if (e != cudaSuccess) return e;
    }
    e = launch_batch_integrate(b, o, stream);
    if (e != cudaSuccess) return e;
  }
  return e;
}

}  // namespace cc
