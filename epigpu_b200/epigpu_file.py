"""The .epigpu packed binary file (src/readplink.c:1145-1181 writer, :1183-1273 reader).

Layout: "epiGPU" (6 bytes), int32 nid, nsnp, npack, remain, nchr, then ped[nid]
(128 bytes), map[nsnp] (88 bytes on LP64), chromosome[nchr] (44 bytes), then
int32[npack1 * nsnp] genotype words. The record layouts are the reference's C structs
(src/readplink.h:17-39) with the x86-64 alignment padding.
"""
import numpy as np

SIGNATURE = b"epiGPU"

PED = np.dtype({"names": ["family", "id", "paternal", "maternal", "sex", "phen"],
                "formats": ["S30", "S30", "S30", "S30", "S1", "<f4"],
                "offsets": [0, 30, 60, 90, 120, 124], "itemsize": 128})
MAP = np.dtype({"names": ["chr", "snpname", "gd", "pd", "allelename"],
                "formats": ["S30", "S30", "<f8", "<i8", "S2"],
                "offsets": [0, 30, 64, 72, 80], "itemsize": 88})
CHROM = np.dtype({"names": ["chrid", "chrname", "chrsize", "chrstart"],
                  "formats": ["<i4", "S30", "<i4", "<i4"],
                  "offsets": [0, 4, 36, 40], "itemsize": 44})


class EpiData:
    def __init__(self, nid, nsnp, npack, remain, ped, genmap, chrom, gpack):
        self.nid, self.nsnp, self.npack, self.remain = nid, nsnp, npack, remain
        self.ped, self.genmap, self.chrom, self.gpack = ped, genmap, chrom, gpack

    @property
    def nchr(self):
        return len(self.chrom)

    def blocks(self):
        """Chromosome blocks (i, j <= i) in perform_scan's order (EpiOpenCL.c:1527-1540)."""
        out = []
        for i in range(self.nchr):
            for j in range(i + 1):
                out.append((int(self.chrom["chrstart"][i]), int(self.chrom["chrsize"][i]),
                            int(self.chrom["chrstart"][j]), int(self.chrom["chrsize"][j])))
        return out


def make(gpack, nid, phen, chrom_sizes, chrom_names=None, snp_names=None):
    """Builds an EpiData from packed genotypes, a phenotype and chromosome sizes."""
    gpack = np.ascontiguousarray(gpack, dtype=np.int32)
    nsnp = gpack.shape[0]
    assert sum(chrom_sizes) == nsnp
    ped = np.zeros(nid, dtype=PED)
    ped["family"] = [str(i + 1).encode() for i in range(nid)]
    ped["id"] = b"1"
    ped["paternal"] = b"0"
    ped["maternal"] = b"0"
    ped["sex"] = b"\x01"
    ped["phen"] = np.asarray(phen, dtype=np.float32)
    genmap = np.zeros(nsnp, dtype=MAP)
    chrom = np.zeros(len(chrom_sizes), dtype=CHROM)
    start = 0
    for c, size in enumerate(chrom_sizes):
        name = (chrom_names[c] if chrom_names else str(c + 1)).encode()
        chrom[c] = (c + 1, name, size, start)
        genmap["chr"][start:start + size] = name
        start += size
    genmap["snpname"] = [(snp_names[s] if snp_names else "rs%d" % (s + 1)).encode() for s in range(nsnp)]
    genmap["pd"] = np.arange(1, nsnp + 1) * 1000
    genmap["allelename"] = b"AG"
    return EpiData(nid, nsnp, nid // 16, nid % 16, ped, genmap, chrom, gpack)


def write(path, d: EpiData):
    with open(path, "wb") as f:
        f.write(SIGNATURE)
        np.array([d.nid, d.nsnp, d.npack, d.remain, d.nchr], dtype="<i4").tofile(f)
        d.ped.astype(PED).tofile(f)
        d.genmap.astype(MAP).tofile(f)
        d.chrom.astype(CHROM).tofile(f)
        np.ascontiguousarray(d.gpack, dtype="<i4").tofile(f)


def read(path) -> EpiData:
    with open(path, "rb") as f:
        if f.read(6) != SIGNATURE:
            raise ValueError("Invalid input file")
        nid, nsnp, npack, remain, nchr = (int(x) for x in np.fromfile(f, dtype="<i4", count=5))
        ped = np.fromfile(f, dtype=PED, count=nid)
        genmap = np.fromfile(f, dtype=MAP, count=nsnp)
        chrom = np.fromfile(f, dtype=CHROM, count=nchr)
        npack1 = npack + (1 if remain else 0)
        gpack = np.fromfile(f, dtype="<i4", count=npack1 * nsnp)
        if len(ped) != nid or len(genmap) != nsnp or len(chrom) != nchr or gpack.size != npack1 * nsnp:
            raise ValueError("truncated .epigpu file")
    return EpiData(nid, nsnp, npack, remain, ped, genmap, chrom, gpack.reshape(nsnp, npack1))
