// rabbit::FileReader (the reference's include/RabbitFX/io/FileReader.h) for the build
// of the reference's own code here, in place of its FileReader.cpp: that file needs
// ISA-L and rapidgzip (absent) even for plain input.  Plain files are read with stdio,
// gzip files with zlib, which is what the header's non-ISA-L configuration describes.
// The reference's record parsing (Formater.cpp, FastxStream.cpp) is unchanged.
// Test and baseline infrastructure only.
#include "RabbitFX/io/FileReader.h"

namespace rabbit {

FileReader::FileReader(const std::string& fileName_, bool isZipped_, const std::size_t) {
    const bool gz = isZipped_ || (fileName_.size() >= 3 && fileName_.compare(fileName_.size() - 3, 3, ".gz") == 0);
    if (gz) {
        isZipped = true;
        mZipFile = gzopen(fileName_.c_str(), "r");
        if (mZipFile == NULL) throw RioException(("Can not open file to read: " + fileName_).c_str());
    } else {
        mFile = FOPEN(fileName_.c_str(), "rb");
        if (mFile == NULL) throw RioException(("Can not open file to read: " + fileName_).c_str());
    }
}

int64 FileReader::Read(byte* memory_, uint64 size_) {
    if (isZipped) {
        const int64 n = gzread(mZipFile, memory_, (unsigned)size_);
        if (n == -1) std::cerr << "Error to read gzip file" << std::endl;
        return n;
    }
    return (int64)fread(memory_, 1, size_, mFile);
}

bool FileReader::FinishRead() { return isZipped ? gzeof(mZipFile) : feof(mFile); }

FileReader::~FileReader() {
    if (mFile != NULL) fclose(mFile);
    if (mZipFile != NULL) gzclose(mZipFile);
}

}  // namespace rabbit
