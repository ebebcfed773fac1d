// holoflow_b200 acquisition files: the .holo container read and written the way Holoflow's
// holofile library does (holofile/include/holofile/holofile.hh:87-152,
// holofile/src/holofile.cc:42-268), restated in namespace hfb::holofile.
//
// Layout (little endian): a 64-byte packed header, frame_count frames of
// width * height * bits_per_pixel / 8 bytes each, then an optional JSON footer holding the
// pipeline settings.  Header fields and their byte offsets:
//   0 magic_number "HOLO" (0x4F4C4F48 read as a little-endian u32) | 4 version (u16, 66)
//   6 bits_per_pixel (u16) | 8 frame_width (u32) | 12 frame_height (u32) | 16 frame_count (u32)
//   20 data_size_in_bytes (u64) | 28 endianness (u8, 0 = little) | 29..63 padding
// Validation follows the reference: a short header is IncompleteHeader, a wrong magic number is
// InvalidMagicNumber, a frame whose bit count is not a whole number of bytes is InvalidFrameSize
// (so 12-bit files need an even pixel count); the footer is read only when the file extends past
// the data, is at most 1 MiB and starts with '{', and a footer that fails those checks or does
// not parse is dropped (footer() is empty) rather than failing the open.
//
// Difference from the reference: where it calls std::exit() on a short fread/fwrite that is not
// end-of-file, this library throws Exception; a library must not end the process.
//
// bits_per_pixel = 12 holds Mono12p frames (2 pixels in 3 bytes, little endian: byte0 = p0[7:0],
// byte1 = p0[11:8] | p1[3:0] << 4, byte2 = p1[11:4]), the camera format of the Doppler path.
#pragma once

#include <cstdint>
#include <cstdio>
#include <memory>
#include <nlohmann/json.hpp>
#include <optional>
#include <stdexcept>
#include <string>

namespace hfb::holofile {

class Exception : public std::runtime_error {
public:
  explicit Exception(const std::string &message) : std::runtime_error(message) {}
};
class EndOfFileException : public Exception {
public:
  EndOfFileException() : Exception("Holofile: End of file reached") {}
};
class IncompleteHeaderException : public Exception {
public:
  IncompleteHeaderException() : Exception("Holofile: Incomplete header") {}
};
class InvalidMagicNumberException : public Exception {
public:
  InvalidMagicNumberException() : Exception("Holofile: Invalid magic number") {}
};
class InvalidVersionException : public Exception {
public:
  InvalidVersionException() : Exception("Holofile: Invalid version") {}
};
class InvalidFrameSizeException : public Exception {
public:
  InvalidFrameSizeException() : Exception("Holofile: Invalid frame size") {}
};
class InvalidFooterException : public Exception {
public:
  InvalidFooterException() : Exception("Holofile: Invalid footer") {}
};

#pragma pack(push, 1)
struct Header {
  uint32_t magic_number       = MAGIC_NUMBER_LE;
  uint16_t version            = CURRENT_VERSION;
  uint16_t bits_per_pixel     = 0;
  uint32_t frame_width        = 0;
  uint32_t frame_height       = 0;
  uint32_t frame_count        = 0;
  uint64_t data_size_in_bytes = 0;
  uint8_t  endianness         = LITTLE_ENDIAN_FILE;
  char     padding[35]        = {};

  static constexpr uint16_t CURRENT_VERSION    = 66;
  static constexpr uint8_t  LITTLE_ENDIAN_FILE = 0;
  static constexpr uint8_t  BIG_ENDIAN_FILE    = 1;
  static constexpr uint32_t MAGIC_NUMBER_LE    = 0x4F4C4F48;

  // bytes of one frame (the reference computes width * height * bits / 8 the same way)
  [[nodiscard]] uint64_t frame_bytes() const {
    return (uint64_t)frame_width * frame_height * bits_per_pixel / 8;
  }
};
#pragma pack(pop)
static_assert(sizeof(Header) == 64, "a .holo header is 64 bytes");

struct Footer {
  nlohmann::json pipeline_settings;
};

class Reader {
public:
  explicit Reader(const std::string &path);
  [[nodiscard]] const Header         &header() const { return header_; }
  [[nodiscard]] std::optional<Footer> footer() const { return footer_; }
  void                                seek(std::size_t frame_index);
  [[nodiscard]] std::size_t           tell() const { return frame_index_; }
  // Reads frame_count frames at the cursor into `data`; EndOfFileException when the file ends
  // first (the frames read so far stay in `data` and the cursor advances past them).
  void read_frames(uint8_t *data, std::size_t frame_count);

private:
  void read_footer();
  struct Closer {
    void operator()(FILE *f) const { std::fclose(f); }
  };
  std::unique_ptr<FILE, Closer> file_;
  Header                        header_{};
  std::optional<Footer>         footer_;
  std::size_t                   frame_index_ = 0;
};

class Writer {
public:
  // Creates (truncates) `path` and writes `header`; frames and the footer follow.
  Writer(const std::string &path, const Header &header, const Footer &footer);
  void                      write_frames(const uint8_t *data, std::size_t frame_count);
  void                      write_footer();
  [[nodiscard]] std::size_t tell() const { return frame_index_; }

private:
  struct Closer {
    void operator()(FILE *f) const { std::fclose(f); }
  };
  std::unique_ptr<FILE, Closer> file_;
  Header                        header_{};
  Footer                        footer_;
  std::size_t                   frame_index_ = 0;
};

// A header for frame_count frames of width x height at bits_per_pixel (8, 12 or 16), with
// data_size_in_bytes filled in (the reference's sink computes it the same way,
// holotask/src/sinks/holofile.cc:97-112).
Header make_header(uint32_t frame_count, uint32_t width, uint32_t height, uint16_t bits_per_pixel);

} // namespace hfb::holofile
