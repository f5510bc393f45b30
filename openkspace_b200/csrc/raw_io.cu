// Acquisition ingest without HDF5 (openkspace-io/src/ismrmrd/reader.rs:15-24,
// acquisition.rs:33-95, header.rs).  The reference reads `/dataset/xml` and the
// rows of `/dataset/data` (AcquisitionHeader, traj, data) from an ISMRMRD
// HDF5 file through libhdf5, which is absent here.  This reader takes the
// same rows serialised one after another, the layout of an ISMRMRD
// acquisition stream:
//
//   "OKSACQ1\0"                       8 bytes
//   u32 xml_len, xml_len bytes        the ISMRMRD XML header
//   u64 n_acq
//   n_acq records:
//     340-byte AcquisitionHeader      little-endian, packed, in the field order
//                                     of acquisition.rs:33-59 (ismrmrd.h)
//     f32 traj[trajectory_dimensions * number_of_samples]
//     f32 data[2 * active_channels * number_of_samples]   [channel][sample], re/im
//
// A first pass reads the headers (seeking over the samples) and lays out the
// complex samples of every record end to end; the samples are then read
// straight into one pinned host buffer, so okscuda_csrss_reconstruct uploads
// them with asynchronous copies.  The XML header is parsed for the fields the
// cs path uses, with the tag-path rules of header.rs:128-206.
#include <cstdio>
#include <string>

#include "ctx.h"

struct okscuda_raw {
    std::vector<okscuda_acq_header> headers;
    okscuda_c64* data = nullptr;
    long long data_len = 0;
    bool pinned = false;
    int enc[3] = {0, 0, 0}, rec[3] = {0, 0, 0};
    int ky_center = 0, kz_center = 0;
    int receiver_channels = 0;
    std::string xml;
};

namespace {

constexpr int kHeaderBytes = 340;

template <class T>
T rd(const uint8_t* p, int off) {
    T v;
    std::memcpy(&v, p + off, sizeof(T));
    return v;
}

// Byte offsets in the packed 340-byte AcquisitionHeader.
constexpr int kFlags = 2, kNumSamples = 34, kActiveChannels = 38, kDiscardPre = 168, kDiscardPost = 170,
              kCenterSample = 172, kTrajDims = 176, kIdx = 242;   // idx: step_1, step_2, average, slice, ..., segment

// header.rs:128-206 on the path of open elements (local names): the fields
// the cs path reads.
void apply_field(const std::vector<std::string>& path, const std::string& text, okscuda_raw* r) {
    auto ends = [&](std::initializer_list<const char*> suf) {
        if (path.size() < suf.size()) return false;
        size_t i = path.size() - suf.size();
        for (const char* s : suf)
            if (path[i++] != s) return false;
        return true;
    };
    auto num = [&]() { return (int)std::strtol(text.c_str(), nullptr, 10); };
    static const char* ax[3] = {"x", "y", "z"};
    for (int a = 0; a < 3; ++a) {
        if (ends({"encoding", "encodedSpace", "matrixSize", ax[a]})) r->enc[a] = num();
        if (ends({"encoding", "reconSpace", "matrixSize", ax[a]})) r->rec[a] = num();
    }
    if (ends({"acquisitionSystemInformation", "receiverChannels"})) r->receiver_channels = num();
    if (path.size() >= 4 && path[path.size() - 4] == "encoding" && path[path.size() - 3] == "encodingLimits" &&
        path.back() == "center") {
        const std::string& sec = path[path.size() - 2];
        if (sec == "kspace_encoding_step_1") r->ky_center = num();
        if (sec == "kspace_encoding_step_2") r->kz_center = num();
    }
}

std::string local_name(const std::string& s) {
    const size_t i = s.rfind(':');
    return i == std::string::npos ? s : s.substr(i + 1);
}

// Start / end / empty tags, declarations and comments; the text between
// tags (trimmed, the five predefined entities unescaped) goes to apply_field.
bool parse_xml(const std::string& x, okscuda_raw* r) {
    std::vector<std::string> path;
    size_t i = 0;
    while (i < x.size()) {
        if (x[i] == '<') {
            if (x.compare(i, 4, "<!--") == 0) {
                const size_t e = x.find("-->", i + 4);
                if (e == std::string::npos) return false;
                i = e + 3;
                continue;
            }
            const size_t e = x.find('>', i);
            if (e == std::string::npos) return false;
            std::string tag = x.substr(i + 1, e - i - 1);
            i = e + 1;
            if (tag.empty() || tag[0] == '?' || tag[0] == '!') continue;
            if (tag[0] == '/') {
                if (!path.empty()) path.pop_back();
                continue;
            }
            const bool empty = tag.back() == '/';
            size_t n = 0;
            while (n < tag.size() && !isspace((unsigned char)tag[n]) && tag[n] != '/') ++n;
            if (!empty) path.push_back(local_name(tag.substr(0, n)));
        } else {
            const size_t e = x.find('<', i);
            std::string t = x.substr(i, (e == std::string::npos ? x.size() : e) - i);
            i = e == std::string::npos ? x.size() : e;
            size_t a = 0, b = t.size();
            while (a < b && isspace((unsigned char)t[a])) ++a;
            while (b > a && isspace((unsigned char)t[b - 1])) --b;
            if (a == b) continue;
            t = t.substr(a, b - a);
            static const char* ents[5][2] = {{"&lt;", "<"}, {"&gt;", ">"}, {"&quot;", "\""}, {"&apos;", "'"},
                                             {"&amp;", "&"}};
            for (auto& en : ents)
                for (size_t p = t.find(en[0]); p != std::string::npos; p = t.find(en[0], p + 1))
                    t.replace(p, std::strlen(en[0]), en[1]);
            apply_field(path, t, r);
        }
    }
    return true;
}

}  // namespace

extern "C" {

int okscuda_raw_open(const char* path, okscuda_raw** out) {
    if (!path || !out) return OKS_EINVAL;
    *out = nullptr;
    FILE* f = std::fopen(path, "rb");
    if (!f) return OKS_EINVAL;
    auto* r = new okscuda_raw();
    int rc = OKS_OK;
    char magic[8];
    uint32_t xml_len = 0;
    uint64_t n = 0;
    std::vector<long long> file_off;   // where each record's samples sit in the file
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "OKSACQ1\0", 8) != 0 ||
        std::fread(&xml_len, 4, 1, f) != 1 || xml_len > (1u << 26))
        rc = OKS_EINVAL;
    if (!rc) {
        r->xml.resize(xml_len);
        if (xml_len && std::fread(&r->xml[0], 1, xml_len, f) != xml_len) rc = OKS_EINVAL;
        if (!rc && std::fread(&n, 8, 1, f) != 1) rc = OKS_EINVAL;
        if (!rc && !parse_xml(r->xml, r)) rc = OKS_EINVAL;
    }
    // pass 1: headers, and the layout of the samples
    for (uint64_t a = 0; a < n && !rc; ++a) {
        uint8_t h[kHeaderBytes];
        if (std::fread(h, 1, kHeaderBytes, f) != (size_t)kHeaderBytes) { rc = OKS_EINVAL; break; }
        okscuda_acq_header q{};
        q.flags = rd<uint64_t>(h, kFlags);
        q.number_of_samples = rd<uint16_t>(h, kNumSamples);
        q.active_channels = rd<uint16_t>(h, kActiveChannels);
        q.discard_pre = rd<uint16_t>(h, kDiscardPre);
        q.discard_post = rd<uint16_t>(h, kDiscardPost);
        q.center_sample = rd<uint16_t>(h, kCenterSample);
        q.kspace_encode_step_1 = rd<uint16_t>(h, kIdx + 0);
        q.kspace_encode_step_2 = rd<uint16_t>(h, kIdx + 2);
        q.slice = rd<uint16_t>(h, kIdx + 6);
        q.segment = rd<uint16_t>(h, kIdx + 16);
        q.data_offset = r->data_len;
        const long long traj = (long long)rd<uint16_t>(h, kTrajDims) * q.number_of_samples;
        const long long ns = (long long)q.active_channels * q.number_of_samples;
        if (std::fseek(f, (long)(4 * traj), SEEK_CUR) != 0) { rc = OKS_EINVAL; break; }
        file_off.push_back(std::ftell(f));
        if (std::fseek(f, (long)(8 * ns), SEEK_CUR) != 0) { rc = OKS_EINVAL; break; }
        r->headers.push_back(q);
        r->data_len += ns;
    }
    // pass 2: the samples, straight into one pinned buffer
    if (!rc && r->data_len > 0) {
        const size_t bytes = sizeof(okscuda_c64) * (size_t)r->data_len;
        void* p = nullptr;
        if (cudaMallocHost(&p, bytes) == cudaSuccess) {
            r->pinned = true;
        } else {
            (void)cudaGetLastError();   // no device: ordinary host memory
            p = std::malloc(bytes);
        }
        r->data = static_cast<okscuda_c64*>(p);
        if (!r->data) rc = OKS_ENOMEM;
        for (size_t a = 0; a < r->headers.size() && !rc; ++a) {
            const auto& q = r->headers[a];
            const size_t ns = (size_t)q.active_channels * q.number_of_samples;
            if (std::fseek(f, (long)file_off[a], SEEK_SET) != 0 ||
                std::fread(r->data + q.data_offset, sizeof(okscuda_c64), ns, f) != ns)
                rc = OKS_EINVAL;
        }
    }
    std::fclose(f);
    if (rc) {
        okscuda_raw_close(r);
        return rc;
    }
    *out = r;
    return OKS_OK;
}

int okscuda_raw_acq_set(const okscuda_raw* r, okscuda_acq_set* out) {
    if (!r || !out) return OKS_EINVAL;
    out->n_acq = (long long)r->headers.size();
    out->headers = r->headers.data();
    out->data = r->data;
    out->data_len = r->data_len;
    out->data_on_device = 0;
    out->enc_x = r->enc[0]; out->enc_y = r->enc[1]; out->enc_z = r->enc[2];
    out->rec_x = r->rec[0]; out->rec_y = r->rec[1]; out->rec_z = r->rec[2];
    out->ky_center = r->ky_center;
    out->kz_center = r->kz_center;
    return OKS_OK;
}

int okscuda_raw_info(const okscuda_raw* r, int* receiver_channels, int* xml_len) {
    if (!r) return OKS_EINVAL;
    if (receiver_channels) *receiver_channels = r->receiver_channels;
    if (xml_len) *xml_len = (int)r->xml.size();
    return OKS_OK;
}

void okscuda_raw_close(okscuda_raw* r) {
    if (!r) return;
    if (r->data) {
        if (r->pinned) cudaFreeHost(r->data);
        else std::free(r->data);
    }
    delete r;
}

}  // extern "C"
