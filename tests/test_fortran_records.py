"""The checkpoint's record layer (dopamine_b200/csrc/host/fortran_records.hpp) on the CPU: records
as gfortran writes sequential unformatted files - a 4-byte length before and after the payload -
and, for payloads above the subrecord limit (2147483639 bytes; a small limit here), subrecords
whose leading marker is negative when more follow and whose trailing marker is negative when one
precedes.  A small C++ driver is compiled against the header and its bytes are checked here."""
import os
import struct
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
HDR = os.path.join(HERE, "..", "dopamine_b200", "csrc", "host")

DRIVER = r"""
#include <cstdio>
#include <cstring>
#include <vector>
#include "fortran_records.hpp"
int main(int argc, char** argv) {
  std::FILE* f = std::fopen(argv[1], "wb");
  int hdr[3] = {7, 8, 9};
  char big[13];
  for (int i = 0; i < 13; ++i) big[i] = (char)('a' + i);
  bool ok = dpm::frec::write_record(f, hdr, sizeof hdr) && dpm::frec::write_record(f, big, 13, 5) &&
            dpm::frec::write_record(f, nullptr, 0);
  std::fclose(f);
  if (!ok) return 2;
  f = std::fopen(argv[1], "rb");
  std::vector<char> r;
  int back[3];
  if (!dpm::frec::read_record_into(f, back, sizeof back) || back[2] != 9) return 3;
  if (!dpm::frec::read_record(f, r) || r.size() != 13 || std::memcmp(r.data(), big, 13)) return 4;
  if (!dpm::frec::read_record(f, r) || !r.empty()) return 5;
  if (dpm::frec::read_record(f, r)) return 6;  // end of file
  std::fclose(f);
  return 0;
}
"""


def test_records_and_subrecords(tmp_path):
    src = tmp_path / "drv.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "drv"
    try:
        subprocess.run(["g++", "-std=c++17", "-O1", "-I", HDR, str(src), "-o", str(exe)], check=True,
                       capture_output=True)
    except (OSError, subprocess.CalledProcessError) as e:
        pytest.skip(f"no host C++ compiler: {e}")
    out = tmp_path / "rec.bin"
    assert subprocess.run([str(exe), str(out)]).returncode == 0
    b = out.read_bytes()
    # record 1: 12 bytes
    assert struct.unpack_from("<i3ii", b, 0) == (12, 7, 8, 9, 12)
    i = 20
    # record 2: 13 bytes in subrecords of 5, 5, 3
    expect = [(-5, 5), (-5, -5), (3, -3)]
    pos = 0
    for head, tail in expect:
        n = abs(head)
        assert struct.unpack_from("<i", b, i)[0] == head
        assert b[i + 4:i + 4 + n] == bytes(range(ord("a") + pos, ord("a") + pos + n))
        assert struct.unpack_from("<i", b, i + 4 + n)[0] == tail
        i += 8 + n
        pos += n
    # record 3: empty
    assert struct.unpack_from("<ii", b, i) == (0, 0)
    assert len(b) == i + 8
