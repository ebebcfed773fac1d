// .holo container (reader / writer) and the "Holofile" source node.
//
// The container follows holofile/src/holofile.cc:42-268; the node follows
// holotask/src/sources/holofile.cc:190-434 (settings keys, inference checks and messages, the
// Live / CPUCached / GPUCached load kinds, max_fps pacing, wrap-around at end_frame, and the
// update() reuse rules), with 12-bit Mono12p files as packed U8 rows.
#include "holoflow_b200/holofile.hh"

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <system_error>
#include <thread>

#include "holoflow_b200/nodes.hh"

namespace hfb::holofile {

namespace {
[[noreturn]] void throw_errno(const std::string &what) {
  throw std::system_error(std::error_code(errno, std::generic_category()), what);
}
constexpr size_t kMaxFooterBytes = 1024 * 1024;
} // namespace

Reader::Reader(const std::string &path) {
  FILE *fp = std::fopen(path.c_str(), "rb");
  if (!fp)
    throw_errno("Failed to open \"" + path + "\"");
  file_.reset(fp);

  const size_t got = std::fread(&header_, sizeof(header_), 1, file_.get());
  if (std::ferror(file_.get()))
    throw_errno("Failed to read header:");
  if (std::feof(file_.get()) || got != 1)
    throw IncompleteHeaderException();
  if (header_.magic_number != Header::MAGIC_NUMBER_LE)
    throw InvalidMagicNumberException();
  // the version field is not checked (the reference leaves version support open)
  if (((uint64_t)header_.frame_width * header_.frame_height * header_.bits_per_pixel) % 8 != 0)
    throw InvalidFrameSizeException();

  try {
    read_footer();
  } catch (const Exception &) {
    footer_.reset();
    if (fseeko(file_.get(), (off_t)sizeof(Header), SEEK_SET) != 0)
      throw_errno("Failed to seek:");
  }
}

void Reader::read_footer() {
  const uint64_t footer_offset = sizeof(Header) + header_.data_size_in_bytes;
  const off_t    current       = ftello(file_.get());
  if (current < 0)
    throw_errno("Failed to get current file position:");
  if (fseeko(file_.get(), 0, SEEK_END) != 0)
    throw_errno("Failed to seek to end:");
  const off_t file_size = ftello(file_.get());
  if (file_size < 0)
    throw_errno("Failed to get file size:");
  if ((uint64_t)file_size <= footer_offset)
    throw InvalidFooterException(); // the file ends with the data: no footer
  const uint64_t footer_size = (uint64_t)file_size - footer_offset;
  if (footer_size > kMaxFooterBytes)
    throw InvalidFooterException();
  if (fseeko(file_.get(), (off_t)footer_offset, SEEK_SET) != 0)
    throw_errno("Failed to seek to footer:");
  std::string text(footer_size, '\0');
  if (std::fread(text.data(), 1, footer_size, file_.get()) != footer_size)
    throw_errno("Failed to read footer:");
  if (text.empty() || text[0] != '{')
    throw InvalidFooterException();
  try {
    footer_ = Footer{nlohmann::json::parse(text)};
  } catch (const nlohmann::json::exception &) {
    throw InvalidFooterException();
  }
  if (fseeko(file_.get(), current, SEEK_SET) != 0)
    throw_errno("Failed to restore file position:");
}

void Reader::seek(std::size_t frame_index) {
  const uint64_t offset = sizeof(Header) + (uint64_t)frame_index * header_.frame_bytes();
  if (fseeko(file_.get(), (off_t)offset, SEEK_SET) != 0)
    throw_errno("Failed to seek:");
  frame_index_ = frame_index;
}

void Reader::read_frames(uint8_t *data, std::size_t frame_count) {
  const size_t fb   = header_.frame_bytes();
  const size_t read = frame_count ? std::fread(data, fb, frame_count, file_.get()) : 0;
  frame_index_ += read;
  if (std::ferror(file_.get()))
    throw_errno("Failed to read frames:");
  if (read != frame_count && std::feof(file_.get()))
    throw EndOfFileException();
  if (read != frame_count)
    throw Exception("Holofile: short read of frames");
}

Writer::Writer(const std::string &path, const Header &header, const Footer &footer)
    : header_(header), footer_(footer) {
  FILE *fp = std::fopen(path.c_str(), "wb");
  if (!fp)
    throw_errno("Failed to open \"" + path + "\"");
  file_.reset(fp);
  const size_t put = std::fwrite(&header_, sizeof(header_), 1, file_.get());
  if (std::ferror(file_.get()))
    throw_errno("Failed to write header:");
  if (put != 1)
    throw Exception("Holofile: short write of the header");
}

void Writer::write_frames(const uint8_t *data, std::size_t frame_count) {
  const size_t fb      = header_.frame_bytes();
  const size_t written = frame_count ? std::fwrite(data, fb, frame_count, file_.get()) : 0;
  frame_index_ += written;
  if (std::ferror(file_.get()))
    throw_errno("Failed to write frames:");
  if (written != frame_count)
    throw Exception("Holofile: short write of frames");
}

void Writer::write_footer() {
  const std::string text = footer_.pipeline_settings.dump();
  if (fseeko(file_.get(), 0, SEEK_END) != 0)
    throw_errno("Failed to seek to end of file:");
  if (std::fwrite(text.data(), 1, text.size(), file_.get()) != text.size())
    throw_errno("Failed to write footer JSON:");
  if (std::fflush(file_.get()) != 0)
    throw_errno("Failed to flush file:");
}

Header make_header(uint32_t frame_count, uint32_t width, uint32_t height, uint16_t bits_per_pixel) {
  Header h;
  h.bits_per_pixel     = bits_per_pixel;
  h.frame_width        = width;
  h.frame_height       = height;
  h.frame_count        = frame_count;
  h.data_size_in_bytes = (uint64_t)frame_count * height * width * bits_per_pixel / 8;
  return h;
}

} // namespace hfb::holofile

// ================================================================================================
// "Holofile" source node
// ================================================================================================
namespace hfb::nodes {

using core::DType;
using core::MemLoc;
using core::OpResult;
using core::SyncCtx;

void from_json(const nlohmann::json &j, HolofileSettings::LoadKind &lk) {
  const auto key = j.get<std::string>();
  if (key == "Live")
    lk = HolofileSettings::LoadKind::Live;
  else if (key == "CPUCached")
    lk = HolofileSettings::LoadKind::CPUCached;
  else if (key == "GPUCached")
    lk = HolofileSettings::LoadKind::GPUCached;
  else
    throw std::invalid_argument("Invalid LoadKind string: " + key);
}

void from_json(const nlohmann::json &j, HolofileSettings &s) {
  j.at("path").get_to(s.path);
  j.at("load_kind").get_to(s.load_kind);
  j.at("start_frame").get_to(s.start_frame);
  j.at("end_frame").get_to(s.end_frame);
  j.at("batch_size").get_to(s.batch_size);
  s.max_fps.reset();
  if (j.contains("max_fps") && !j.at("max_fps").is_null())
    s.max_fps = j.at("max_fps").get<int>();
  s.keep_cursor = j.value("keep_cursor", true);
}

namespace {

void check(bool ok, const std::string &msg) {
  if (!ok)
    throw std::invalid_argument("HolofileFactory inference error: " + msg);
}

void cuda_ok(cudaError_t e, const char *what) {
  if (e != cudaSuccess)
    throw core::CudaError(std::string("Holofile: ") + what + ": " + cudaGetErrorString(e));
}

// [batch, H, W] frames of the file's pixel type; 12-bit files give their packed rows as bytes
TDesc output_desc(const HolofileSettings &s, const holofile::Header &h) {
  const MemLoc loc = s.load_kind == HolofileSettings::LoadKind::GPUCached ? MemLoc::Device : MemLoc::Host;
  if (h.bits_per_pixel == 12)
    return TDesc({(size_t)s.batch_size, h.frame_height, (size_t)h.frame_width * 3 / 2}, DType::U8, loc);
  return TDesc({(size_t)s.batch_size, h.frame_height, h.frame_width}, h.bits_per_pixel == 8 ? DType::U8 : DType::U16,
               loc);
}

class HolofileTask final : public ISyncTask {
public:
  using Clock = std::chrono::steady_clock;

  HolofileSettings                  settings;
  std::unique_ptr<holofile::Reader> reader;
  holofile::Header                  header{};
  int                               frame_idx = 0;
  TDesc                             odesc;
  std::optional<Clock::time_point>  next_batch_start;
  std::byte                        *buf      = nullptr; // cached frames start_frame .. end_frame
  std::byte                        *h_buf    = nullptr; // CPUCached: pinned when a device exists
  bool                              h_pinned = false;
  std::byte                        *d_buf    = nullptr; // GPUCached
  core::Storage                     published{};        // the view handed out for cached kinds

  ~HolofileTask() override {
    if (d_buf)
      cudaFree(d_buf);
    if (h_buf) {
      if (h_pinned)
        cudaFreeHost(h_buf);
      else
        std::free(h_buf);
    }
  }

  // Waits until this batch's slot when max_fps is set; false if the run was cancelled meanwhile.
  bool pace_before_batch(SyncCtx &ctx) {
    if (!settings.max_fps) {
      next_batch_start.reset();
      return true;
    }
    auto period = std::chrono::duration_cast<Clock::duration>(
        std::chrono::duration<double>((double)settings.batch_size / *settings.max_fps));
    if (period <= Clock::duration::zero())
      period = Clock::duration{1};
    if (!next_batch_start)
      next_batch_start = Clock::now();
    while (Clock::now() < *next_batch_start) {
      if (ctx.cancelled && ctx.cancelled->load(std::memory_order_relaxed))
        return false;
      std::this_thread::yield();
    }
    do
      *next_batch_start += period;
    while (*next_batch_start < Clock::now());
    return true;
  }

  OpResult execute(SyncCtx &ctx) override {
    if (!pace_before_batch(ctx))
      return OpResult::Cancelled;
    const size_t fb = header.frame_bytes();
    if (frame_idx + settings.batch_size > settings.end_frame) { // loop back to start_frame
      if (settings.load_kind == HolofileSettings::LoadKind::Live)
        reader->seek(settings.start_frame);
      frame_idx = settings.start_frame;
    }
    if (settings.load_kind == HolofileSettings::LoadKind::Live) {
      auto *dst = reinterpret_cast<uint8_t *>(ctx.outputs[0].data());
      if (dst == nullptr)
        throw std::invalid_argument("Holofile: a Live source writes into the caller's output buffer");
      reader->read_frames(dst, settings.batch_size);
    } else {
      published      = core::Storage{odesc.mem_loc, odesc.num_bytes(),
                                     buf + (size_t)(frame_idx - settings.start_frame) * fb};
      ctx.outputs[0] = core::TView{odesc, &published};
    }
    frame_idx += settings.batch_size;
    return OpResult::Ok;
  }
};

} // namespace

InferResult HolofileFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const auto             s = j.get<HolofileSettings>();
  const holofile::Reader reader(s.path);
  const auto            &h = reader.header();
  check(input_descs.empty(), "Holofile task must have no inputs");
  check(s.start_frame < s.end_frame, "Invalid frame range");
  check(s.batch_size > 0, "Batch size must be positive");
  check(!s.max_fps || *s.max_fps > 0, "max_fps must be positive when provided");
  check(s.end_frame <= (int64_t)h.frame_count, "end_frame exceeds total frames in file");
  check(s.batch_size <= s.end_frame - s.start_frame, "Batch size exceeds available frames");
  check(h.bits_per_pixel == 8 || h.bits_per_pixel == 12 || h.bits_per_pixel == 16,
        "Unsupported bits_per_pixel: " + std::to_string(h.bits_per_pixel));
  check(h.bits_per_pixel != 12 || h.frame_width % 2 == 0, "12-bit frames need an even frame width");
  InferResult r;
  r.output_descs  = {output_desc(s, h)};
  r.owned_outputs = {s.load_kind != HolofileSettings::LoadKind::Live};
  return r;
}

std::unique_ptr<ISyncTask> HolofileFactory::create(std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                   const SyncCreateCtx &ctx) const {
  const auto inf = infer(input_descs, j);
  auto       t   = std::make_unique<HolofileTask>();
  t->settings    = j.get<HolofileSettings>();
  t->reader      = std::make_unique<holofile::Reader>(t->settings.path);
  t->header      = t->reader->header();
  t->odesc       = inf.output_descs[0];
  t->frame_idx   = t->settings.start_frame;
  t->reader->seek(t->settings.start_frame);
  const size_t fb     = t->header.frame_bytes();
  const size_t frames = (size_t)(t->settings.end_frame - t->settings.start_frame);
  const size_t bytes  = frames * fb;
  switch (t->settings.load_kind) {
  case HolofileSettings::LoadKind::Live:
    break;
  case HolofileSettings::LoadKind::CPUCached: {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0 &&
        cudaHostAlloc(reinterpret_cast<void **>(&t->h_buf), bytes, cudaHostAllocDefault) == cudaSuccess) {
      t->h_pinned = true;
    } else {
      (void)cudaGetLastError();
      t->h_buf = static_cast<std::byte *>(std::malloc(bytes));
      if (!t->h_buf)
        throw std::bad_alloc();
    }
    t->reader->read_frames(reinterpret_cast<uint8_t *>(t->h_buf), frames);
    t->buf = t->h_buf;
  } break;
  case HolofileSettings::LoadKind::GPUCached: {
    cuda_ok(cudaMalloc(reinterpret_cast<void **>(&t->d_buf), bytes), "device cache");
    // stream the file through a bounded pinned staging buffer
    const size_t chunk_frames =
        std::max<size_t>(1, std::min(frames, (size_t)(64u << 20) / std::max<size_t>(fb, 1)));
    std::byte *stage = nullptr;
    cuda_ok(cudaHostAlloc(reinterpret_cast<void **>(&stage), chunk_frames * fb, cudaHostAllocDefault), "staging");
    try {
      for (size_t f = 0; f < frames; f += chunk_frames) {
        const size_t n = std::min(chunk_frames, frames - f);
        t->reader->read_frames(reinterpret_cast<uint8_t *>(stage), n);
        cuda_ok(cudaMemcpyAsync(t->d_buf + f * fb, stage, n * fb, cudaMemcpyHostToDevice, ctx.stream), "upload");
        cuda_ok(cudaStreamSynchronize(ctx.stream), "upload"); // the staging buffer is reused next
      }
    } catch (...) {
      cudaFreeHost(stage);
      throw;
    }
    cudaFreeHost(stage);
    t->buf = t->d_buf;
  } break;
  }
  return t;
}

std::unique_ptr<ISyncTask> HolofileFactory::update(std::unique_ptr<ISyncTask> old, std::span<const TDesc> input_descs,
                                                   const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  auto *o = dynamic_cast<HolofileTask *>(old.get());
  if (!o)
    return create(input_descs, j, ctx);
  const auto inf         = infer(input_descs, j);
  const auto s           = j.get<HolofileSettings>();
  const bool live        = s.load_kind == HolofileSettings::LoadKind::Live;
  const bool bounds_same = o->settings.start_frame == s.start_frame && o->settings.end_frame == s.end_frame;
  const bool can_reuse   = o->settings.path == s.path && o->settings.load_kind == s.load_kind && (live || bounds_same);
  if (!can_reuse) {
    old.reset();
    return create(input_descs, j, ctx);
  }
  int frame_idx = s.start_frame;
  if (s.keep_cursor) {
    frame_idx = o->frame_idx;
    if (frame_idx < s.start_frame || frame_idx >= s.end_frame) // bounds shrank past the cursor
      frame_idx = s.start_frame;
  }
  if (live && frame_idx != o->frame_idx)
    o->reader->seek(frame_idx);
  const bool pace_same = o->settings.batch_size == s.batch_size && o->settings.max_fps == s.max_fps;
  o->settings          = s;
  o->odesc             = inf.output_descs[0];
  o->frame_idx         = frame_idx;
  if (!pace_same)
    o->next_batch_start.reset();
  return old;
}

} // namespace hfb::nodes
