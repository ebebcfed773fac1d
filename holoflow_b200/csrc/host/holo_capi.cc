// C ABI over the .holo reader / writer (holoflow_b200/holofile.hh).  Exceptions become statuses:
// a malformed file (holofile::Exception other than end of file) is HF_ERR_INVALID, reading past
// the last frame and I/O failures are HF_ERR_STATE; the message is in hf_last_error().
#include <cstring>

#include "hf_common.cuh"
#include "holoflow_b200.h"
#include "holoflow_b200/holofile.hh"

using namespace hfb;

static_assert(sizeof(hf_holo_header) == sizeof(holofile::Header), "hf_holo_header is the file's 64-byte header");

struct hf_holo_reader {
  std::unique_ptr<holofile::Reader> r;
};
struct hf_holo_writer {
  std::unique_ptr<holofile::Writer> w;
};

namespace {
template <class F> int guarded(F &&f) {
  hf::clear_error();
  try {
    return f();
  } catch (const holofile::EndOfFileException &e) {
    return hf::fail(HF_ERR_STATE, e.what());
  } catch (const holofile::Exception &e) {
    return hf::fail(HF_ERR_INVALID, e.what());
  } catch (const nlohmann::json::exception &e) {
    return hf::fail(HF_ERR_INVALID, std::string("footer: ") + e.what());
  } catch (const std::invalid_argument &e) {
    return hf::fail(HF_ERR_INVALID, e.what());
  } catch (const std::exception &e) {
    return hf::fail(HF_ERR_STATE, e.what());
  }
}
} // namespace

extern "C" {

int hf_holo_open(const char *path, hf_holo_reader **reader) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(path != nullptr && reader != nullptr, "hf_holo_open: null argument");
    *reader = nullptr;
    auto h  = std::make_unique<hf_holo_reader>();
    h->r    = std::make_unique<holofile::Reader>(path);
    *reader = h.release();
    return HF_OK;
  });
}

int hf_holo_header_get(const hf_holo_reader *reader, hf_holo_header *header) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(reader != nullptr && header != nullptr, "hf_holo_header_get: null argument");
    std::memcpy(header, &reader->r->header(), sizeof(hf_holo_header));
    return HF_OK;
  });
}

int hf_holo_footer(const hf_holo_reader *reader, char *buf, size_t cap, size_t *len) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(reader != nullptr && len != nullptr, "hf_holo_footer: null argument");
    const auto        f    = reader->r->footer();
    const std::string text = f ? f->pipeline_settings.dump() : std::string();
    *len                   = text.size();
    if (buf) {
      HF_CHECK_ARG(cap > text.size(), "hf_holo_footer: buffer too small");
      std::memcpy(buf, text.c_str(), text.size() + 1);
    }
    return HF_OK;
  });
}

int hf_holo_seek(hf_holo_reader *reader, int64_t frame_index) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(reader != nullptr && frame_index >= 0, "hf_holo_seek: bad argument");
    reader->r->seek((size_t)frame_index);
    return HF_OK;
  });
}

int hf_holo_tell(const hf_holo_reader *reader, int64_t *frame_index) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(reader != nullptr && frame_index != nullptr, "hf_holo_tell: null argument");
    *frame_index = (int64_t)reader->r->tell();
    return HF_OK;
  });
}

int hf_holo_read(hf_holo_reader *reader, void *dst, int64_t count) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(reader != nullptr && count >= 0 && (dst != nullptr || count == 0), "hf_holo_read: bad argument");
    reader->r->read_frames(static_cast<uint8_t *>(dst), (size_t)count);
    return HF_OK;
  });
}

int hf_holo_close(hf_holo_reader *reader) {
  return guarded([&]() -> int {
    delete reader;
    return HF_OK;
  });
}

int hf_holo_create(const char *path, uint32_t frame_count, uint32_t width, uint32_t height, uint16_t bits_per_pixel,
                   const char *footer_json, hf_holo_writer **writer) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(path != nullptr && writer != nullptr, "hf_holo_create: null argument");
    HF_CHECK_ARG(bits_per_pixel == 8 || bits_per_pixel == 12 || bits_per_pixel == 16,
                 "hf_holo_create: bits_per_pixel must be 8, 12 or 16");
    HF_CHECK_ARG(((uint64_t)width * height * bits_per_pixel) % 8 == 0,
                 "hf_holo_create: a frame must be a whole number of bytes");
    *writer = nullptr;
    holofile::Footer footer{footer_json && *footer_json ? nlohmann::json::parse(footer_json)
                                                        : nlohmann::json::object()};
    auto h = std::make_unique<hf_holo_writer>();
    h->w   = std::make_unique<holofile::Writer>(path, holofile::make_header(frame_count, width, height, bits_per_pixel),
                                              footer);
    *writer = h.release();
    return HF_OK;
  });
}

int hf_holo_write(hf_holo_writer *writer, const void *src, int64_t count) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(writer != nullptr && writer->w != nullptr && count >= 0 && (src != nullptr || count == 0),
                 "hf_holo_write: bad argument");
    writer->w->write_frames(static_cast<const uint8_t *>(src), (size_t)count);
    return HF_OK;
  });
}

int hf_holo_finish(hf_holo_writer *writer) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(writer != nullptr, "hf_holo_finish: null argument");
    std::unique_ptr<hf_holo_writer> owned(writer);
    if (owned->w)
      owned->w->write_footer();
    return HF_OK;
  });
}

} // extern "C"
