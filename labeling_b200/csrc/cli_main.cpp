// cli_main.cpp -- `labeling`, the command line of the reference's demo (Labeling2015/main.cpp)
// on the B200 labeler.
//
//   labeling -a bleq -g -i <image | dir> [-o <dir>] [-l cycles] [-c 4|8]
//   labeling -a bleq -3 -g -i <slice dir | volume.npy> [-o <dir>] [-l cycles]
//
// Same keys as the reference (ParseInput, main.cpp:399-447): -i -o -a -3 -g -u -j -l -c -h.
// Images are read without OpenCV: binary PGM / PPM (P5 / P6) and uint8 .npy (2D, or 3D volumes with
// the last axis fastest).  A 3D slice directory is read like Read3DImage (main.cpp:172-212): sorted
// slice files, each binarized, stacked with the slice index as the fastest axis.  -o writes colour
// label images as PPM (LabelsToRGB / Write3DLabels, main.cpp:272-305; fixed-seed colours).
#include "labeling.hpp"

#include <algorithm>
#include <array>
#include <cctype>
#include <climits>
#include <cstdio>
#include <cstring>
#include <dirent.h>
#include <iomanip>
#include <iostream>
#include <map>
#include <random>
#include <sstream>
#include <sys/stat.h>

using namespace LabelingB200;

namespace {

struct Options {
    std::string inPath, outPath, algName;
    int numThreads = MAX_THREADS, cycles = 1;
    enum { OCL_NO, OCL_CPU, OCL_GPU } useGPU = OCL_NO;
    TCoherence coh = COH_DEFAULT;
    bool label3D = false, quickExit = false;
};

// Min / avg / max of the -l cycles (ImgTime, main.cpp:46-84).
struct ImgTime {
    TTime mn = UINT_MAX, mx = 0;
    double sum = 0;
    size_t c = 0;
    void Add(TTime t) { mn = std::min(mn, t); mx = std::max(mx, t); sum += t; ++c; }
    void Merge(const ImgTime &o) { mn = std::min(mn, o.mn); mx = std::max(mx, o.mx); sum += o.sum; c += o.c; }
    double Min() const { return c ? mn : 0; }
    double Avg() const { return c ? sum / c : 0; }
    double Max() const { return mx; }
};

bool is_dir(const std::string &p)
{
    struct stat st;
    return stat(p.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

bool exists(const std::string &p)
{
    struct stat st;
    return stat(p.c_str(), &st) == 0;
}

std::string ext_of(const std::string &p)
{
    const size_t d = p.rfind('.');
    std::string e = d == std::string::npos ? "" : p.substr(d);
    std::transform(e.begin(), e.end(), e.begin(), ::tolower);
    return e;
}

std::string file_name(const std::string &p)
{
    const size_t s = p.rfind('/');
    return s == std::string::npos ? p : p.substr(s + 1);
}

std::vector<std::string> find_files(const std::string &dir)
{
    static const char *exts[] = {".pgm", ".ppm", ".npy"};
    std::vector<std::string> out;
    DIR *d = opendir(dir.c_str());
    if (!d) return out;
    while (dirent *e = readdir(d)) {
        const std::string f = dir + "/" + e->d_name;
        if (is_dir(f)) continue;
        const std::string x = ext_of(f);
        for (const char *k : exts)
            if (x == k) out.push_back(f);
    }
    closedir(d);
    std::sort(out.begin(), out.end());
    return out;
}

// ---- image I/O ---------------------------------------------------------------------------------
TImage read_pnm(const std::string &path)
{
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) throw Error(BE_ERR_INVALID, "Cannot open " + path);
    char magic[3] = {0};
    int w = 0, h = 0, maxv = 0;
    if (std::fscanf(f, "%2s", magic) != 1) { std::fclose(f); throw Error(BE_ERR_INVALID, "Bad image " + path); }
    auto skip = [&]() {
        int c;
        while ((c = std::fgetc(f)) != EOF) {
            if (c == '#') { while ((c = std::fgetc(f)) != EOF && c != '\n') {} }
            else if (!std::isspace(c)) { std::ungetc(c, f); break; }
        }
    };
    skip();
    bool ok = std::fscanf(f, "%d", &w) == 1;
    skip();
    ok = ok && std::fscanf(f, "%d", &h) == 1;
    skip();
    ok = ok && std::fscanf(f, "%d", &maxv) == 1;
    std::fgetc(f);
    if (!ok) { std::fclose(f); throw Error(BE_ERR_INVALID, "Bad image header " + path); }
    const int ch = std::strcmp(magic, "P6") == 0 ? 3 : std::strcmp(magic, "P5") == 0 ? 1 : 0;
    if (!ch || w <= 0 || h <= 0 || maxv != 255) { std::fclose(f); throw Error(BE_ERR_INVALID, "Unsupported image " + path); }
    TImage img;
    img.dims = 2; img.size[0] = h; img.size[1] = w; img.channels = ch;
    img.data.resize(size_t(w) * h * ch);
    const size_t got = std::fread(img.data.data(), 1, img.data.size(), f);
    std::fclose(f);
    if (got != img.data.size()) throw Error(BE_ERR_INVALID, "Truncated image " + path);
    return img;
}

TImage read_npy(const std::string &path)
{
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) throw Error(BE_ERR_INVALID, "Cannot open " + path);
    char pre[10];
    if (std::fread(pre, 1, 10, f) != 10 || std::memcmp(pre, "\x93NUMPY", 6) != 0) {
        std::fclose(f);
        throw Error(BE_ERR_INVALID, "Not a .npy file: " + path);
    }
    size_t hlen = size_t(uint8_t(pre[8])) | (size_t(uint8_t(pre[9])) << 8);
    if (pre[6] >= 2) {   // version 2+: 4-byte header length
        unsigned char b[2];
        if (std::fread(b, 1, 2, f) != 2) { std::fclose(f); throw Error(BE_ERR_INVALID, "Truncated .npy: " + path); }
        hlen = hlen | (size_t(b[0]) << 16) | (size_t(b[1]) << 24);
    }
    std::string hdr(hlen, ' ');
    if (std::fread(&hdr[0], 1, hlen, f) != hlen) { std::fclose(f); throw Error(BE_ERR_INVALID, "Truncated .npy: " + path); }
    if (hdr.find("'|u1'") == std::string::npos || hdr.find("'fortran_order': False") == std::string::npos) {
        std::fclose(f);
        throw Error(BE_ERR_INVALID, "Only C-ordered uint8 .npy arrays are supported: " + path);
    }
    const size_t a = hdr.find('(', hdr.find("'shape'")), b = hdr.find(')', a);
    std::vector<int> shape;
    std::stringstream ss(hdr.substr(a + 1, b - a - 1));
    std::string tok;
    while (std::getline(ss, tok, ','))
        if (tok.find_first_not_of(' ') != std::string::npos) shape.push_back(std::stoi(tok));
    TImage img;
    if (shape.size() == 2) { img.dims = 2; img.size[0] = shape[0]; img.size[1] = shape[1]; }
    else if (shape.size() == 3) { img.dims = 3; for (int i = 0; i < 3; ++i) img.size[i] = shape[i]; }
    else { std::fclose(f); throw Error(BE_ERR_INVALID, "Unsupported .npy shape: " + path); }
    img.data.resize(img.total());
    const size_t got = std::fread(img.data.data(), 1, img.data.size(), f);
    std::fclose(f);
    if (got != img.data.size()) throw Error(BE_ERR_INVALID, "Truncated .npy: " + path);
    return img;
}

TImage read_image(const std::string &path) { return ext_of(path) == ".npy" ? read_npy(path) : read_pnm(path); }

// LabelsToRGB (main.cpp:250-286) with a fixed-seed colour per label, background black.
void write_labels_ppm(const std::string &path, const TLabel *lab, int rows, int cols,
                      std::map<TLabel, std::array<uint8_t, 3>> &colors, std::mt19937 &rng)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) throw Error(BE_ERR_INVALID, "Cannot write " + path);
    std::fprintf(f, "P6\n%d %d\n255\n", cols, rows);
    std::vector<uint8_t> row(size_t(cols) * 3);
    for (int y = 0; y < rows; ++y) {
        for (int x = 0; x < cols; ++x) {
            const TLabel l = lab[size_t(y) * cols + x];
            std::array<uint8_t, 3> c = {0, 0, 0};
            if (l) {
                auto it = colors.find(l);
                if (it == colors.end())
                    it = colors.emplace(l, std::array<uint8_t, 3>{uint8_t(rng()), uint8_t(rng()), uint8_t(rng())}).first;
                c = it->second;
            }
            std::memcpy(&row[3 * size_t(x)], c.data(), 3);
        }
        std::fwrite(row.data(), 1, row.size(), f);
    }
    std::fclose(f);
}

void PrintHelp()
{
    std::cout << "Usage: labeling [options]\n\n"
                 "Options:\n"
                 "  -i <input_path> : Input file or path (PGM/PPM/.npy; 3D: slice directory or .npy)\n"
                 "  -o <out_path>   : Output path\n"
                 "  -a <algorithm>  : Labeling algorithm:\n";
    for (const auto &a : AlgList())
        std::cout << std::setw(12) << ' ' << std::setw(9) << std::left << a.first << ": " << a.second.descr
                  << " (" << (a.second.cpu ? "CPU" : "") << (a.second.cpu3d ? "+3D" : "")
                  << (a.second.gpu ? " GPU" : "") << (a.second.gpu3d ? "+3D" : "") << ")\n";
    std::cout << "  -3           : Treat input sequence as a single 3D image\n"
                 "  -g           : Run algorithm on the GPU\n"
                 "  -u           : (OpenCL on CPU in the reference; not available)\n"
                 "  -j <threads> : Number of host threads (accepted, unused)\n"
                 "  -l <cycles>  : Number of cycles for each image (default 1)\n"
                 "  -c <connect> : Connectivity (4 or 8 [default]); block equivalence supports 8\n"
                 "  -h           : Print this help\n\n";
}

Options ParseInput(int argc, char **argv)
{
    Options o;
    auto data = [&](int &i) -> std::string {
        if (i + 1 < argc) return argv[++i];
        throw Error(BE_ERR_INVALID, std::string("Wrong input parameters (no data following the key ") + argv[i] + ")");
    };
    for (int i = 1; i < argc; ++i) {
        const std::string k = argv[i];
        if (k == "-i") { o.inPath = data(i); continue; }
        if (k == "-o") { o.outPath = data(i); continue; }
        if (k == "-a") { o.algName = data(i); continue; }
        if (k == "-3") { o.label3D = true; continue; }
        if (k == "-g") { o.useGPU = Options::OCL_GPU; continue; }
        if (k == "-u") { o.useGPU = Options::OCL_CPU; continue; }
        if (k == "-j") { o.numThreads = std::stoi(data(i)); continue; }
        if (k == "-l") { o.cycles = std::stoi(data(i)); continue; }
        if (k == "-c") { o.coh = data(i) == "4" ? COH_4 : COH_8; continue; }
        if (k == "-h") { PrintHelp(); o.quickExit = true; return o; }
        throw Error(BE_ERR_INVALID, "Wrong input parameters (unknown key " + k + ")");
    }
    return o;
}

TLabelImage LabelCycles(ILabeling &alg, const TImage &img, const Options &o, ImgTime &t)
{
    TLabelImage labels;
    for (int c = 0; c < std::max(1, o.cycles); ++c) t.Add(alg.Label(img, labels, char(o.numThreads), o.coh));
    return labels;
}

void PrintTime(const std::string &name, const ImgTime &t, const Options &o)
{
    std::cout << "Image: " << name << "\n";
    if (o.cycles <= 1) std::cout << "Processing time: " << t.Avg() / 1000 << " ms\n";
    else std::cout << "Processing time:\n Min = " << t.Min() / 1000 << "ms\n Avg = " << t.Avg() / 1000
                   << "ms\n Max = " << t.Max() / 1000 << "ms\n";
}

void Run(const Options &o)
{
    if (o.useGPU == Options::OCL_CPU)
        throw Error(BE_ERR_INVALID, "Chosen algorithm doesn't support specified capabilities (-u: no CPU mode)");
    auto alg = SetLabelingAlg(o.algName, o.useGPU == Options::OCL_GPU, o.label3D);
    std::mt19937 rng(2016);
    std::map<TLabel, std::array<uint8_t, 3>> colors;
    if (!o.label3D) {
        std::vector<std::string> files = is_dir(o.inPath) ? find_files(o.inPath) : std::vector<std::string>{o.inPath};
        if (!is_dir(o.inPath) && !exists(o.inPath)) { PrintHelp(); throw Error(BE_ERR_INVALID, "Wrong input path"); }
        ImgTime total;
        size_t count = 0;
        for (const std::string &f : files) {
            TImage img = read_image(f);
            if (img.dims != 2) throw Error(BE_ERR_INVALID, "Not a 2D image: " + f + " (use -3)");
            ImgTime t;
            TLabelImage lab = LabelCycles(*alg, img, o, t);
            total.Merge(t);
            if (files.size() > 1)
                std::cout << "Processing image " << ++count << "/" << files.size() << " (" << file_name(f) << ") "
                          << t.Avg() / 1000 << " ms\n";
            else PrintTime(file_name(f), t, o);
            if (!o.outPath.empty() && is_dir(o.outPath)) {
                colors.clear();
                write_labels_ppm(o.outPath + "/" + file_name(f) + ".ppm", lab.data.data(), lab.rows(), lab.cols(),
                                 colors, rng);
            }
        }
        if (files.size() > 1)
            std::cout << "\nMin processing time: " << total.Min() / 1000 << " ms\nAvg processing time: "
                      << total.Avg() / 1000 << " ms\nMax processing time: " << total.Max() / 1000 << " ms\n";
        return;
    }
    // 3D: a .npy volume, or a directory of slices stacked like Read3DImage (slice index fastest).
    TImage vol;
    if (!is_dir(o.inPath)) {
        if (ext_of(o.inPath) != ".npy") { PrintHelp(); throw Error(BE_ERR_INVALID, "Wrong input path (assumed directory with 3D image slices)"); }
        vol = read_npy(o.inPath);
        if (vol.dims != 3) throw Error(BE_ERR_INVALID, "Not a 3D volume: " + o.inPath);
    } else {
        std::vector<std::string> files = find_files(o.inPath);
        int plane = 0;
        for (const std::string &f : files) {
            TImage s = ILabeling::RGB2Gray(read_image(f));
            if (vol.empty()) {
                vol.dims = 3; vol.size[0] = s.rows(); vol.size[1] = s.cols(); vol.size[2] = int(files.size());
                vol.data.assign(vol.total(), 0);
            }
            if (s.rows() != vol.size[0] || s.cols() != vol.size[1])
                throw Error(BE_ERR_INVALID, "Cannot read 3D image: slice sizes do not match");
            for (int i = 0; i < s.rows(); ++i)
                for (int j = 0; j < s.cols(); ++j)
                    vol.data[(size_t(i) * vol.size[1] + j) * vol.size[2] + plane] = s.data[size_t(i) * s.cols() + j];
            ++plane;
        }
        if (vol.empty()) throw Error(BE_ERR_INVALID, "No slices in " + o.inPath);
    }
    ImgTime t;
    TLabelImage lab = LabelCycles(*alg, vol, o, t);
    PrintTime(o.inPath, t, o);
    if (!o.outPath.empty() && is_dir(o.outPath)) {   // Write3DLabels: one image per plane
        std::vector<TLabel> plane(size_t(lab.size[0]) * lab.size[1]);
        for (int p = 0; p < lab.size[2]; ++p) {
            for (int i = 0; i < lab.size[0]; ++i)
                for (int j = 0; j < lab.size[1]; ++j)
                    plane[size_t(i) * lab.size[1] + j] = lab.data[(size_t(i) * lab.size[1] + j) * lab.size[2] + p];
            write_labels_ppm(o.outPath + "/" + std::to_string(p + 1) + ".ppm", plane.data(), lab.size[0], lab.size[1],
                             colors, rng);
        }
    }
}

}  // namespace

int main(int argc, char **argv)
{
    try {
        Options o = ParseInput(argc, argv);
        if (!o.quickExit) Run(o);
    } catch (const std::exception &e) {
        std::cout << "Error: " << e.what() << "\n\n";   // the reference reports and exits 0
    }
    return 0;
}
