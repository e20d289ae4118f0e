/*
 * adb_oracle.c -- TEST INFRASTRUCTURE ONLY (see adb_oracle.h).
 *
 * Single-threaded C restatements of the reference's join kernels.  Each
 * function cites the reference file:line it follows (paths are relative to the
 * AllianceDB source tree).  The multithreaded reference splits the same work
 * across pthreads; the set of matched pairs, and so the count and checksum, do
 * not depend on that split.
 *
 * Deviation kept on purpose: keys are compared as unsigned 32-bit values
 * everywhere.  The reference stores keys as int32 (hashing/utils/types.h:50-51)
 * and its AVX sort compares tuples as doubles (sorting/main.cpp:31-45), so
 * keys >= 2^31 sort wrongly there; for keys < 2^31 both orders agree.
 */
#include "adb_oracle.h"

#include <stdlib.h>
#include <string.h>

uint64_t ora_fmix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

uint64_t ora_pair_hash(uint32_t key, uint32_t r_payload, uint32_t s_payload) {
    uint64_t a = ((uint64_t)key << 32) | r_payload;
    uint64_t b = ((uint64_t)s_payload << 32) | key;
    return ora_fmix64(a ^ ora_fmix64(b));
}

static inline void emit(ora_result *res, uint32_t key, uint32_t rp, uint32_t sp) {
    res->count += 1;
    res->checksum += ora_pair_hash(key, rp, sp);
}

/* NEXT_POW_2 of hashing/joins/parallel_radix_join.cpp:76-86 (v >= 1). */
static uint64_t next_pow2(uint64_t v) {
    uint64_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

/* ------------------------------------------------------------------ */
/* Radix clustering: hashing/joins/parallel_radix_join.cpp:573-614.   */
/* idx = (key & (((1<<D)-1) << R)) >> R; histogram, prefix, scatter.  */
/* Padding between clusters (:600) only spaces the output; omitted.   */
/* ------------------------------------------------------------------ */
static void radix_cluster(ora_tuple *out, const ora_tuple *in, uint64_t n,
                          uint64_t *hist, int R, int D) {
    uint32_t fan = 1u << D;
    uint32_t M = (fan - 1u) << R;
    uint64_t *dst = (uint64_t *)malloc(sizeof(uint64_t) * fan);
    memset(hist, 0, sizeof(uint64_t) * fan);
    for (uint64_t i = 0; i < n; i++) hist[(in[i].key & M) >> R]++;
    uint64_t off = 0;
    for (uint32_t i = 0; i < fan; i++) { dst[i] = off; off += hist[i]; }
    for (uint64_t i = 0; i < n; i++) out[dst[(in[i].key & M) >> R]++] = in[i];
    free(dst);
}

/* Two-pass partitioning of prj_thread (:1089-1108 pass 1, :1217-1219 pass 2):
 * pass 1 on the low NUM_RADIX_BITS/2 bits, pass 2 on the next bits
 * (prj_params.h:75-86).  Returns offsets of the 2^bits final partitions. */
static ora_tuple *two_pass_partition(const ora_tuple *in, uint64_t n, int bits, uint64_t *offs) {
    int b1 = bits / 2, b2 = bits - b1;
    uint32_t f1 = 1u << b1, f2 = 1u << b2;
    ora_tuple *tmp = (ora_tuple *)malloc(sizeof(ora_tuple) * (n ? n : 1));
    ora_tuple *out = (ora_tuple *)malloc(sizeof(ora_tuple) * (n ? n : 1));
    uint64_t *h1 = (uint64_t *)malloc(sizeof(uint64_t) * f1);
    uint64_t *h2 = (uint64_t *)malloc(sizeof(uint64_t) * f2);
    radix_cluster(tmp, in, n, h1, 0, b1);
    uint64_t base = 0;
    for (uint32_t p = 0; p < f1; p++) {
        radix_cluster(out + base, tmp + base, h1[p], h2, b1, b2);
        uint64_t o = base;
        for (uint32_t q = 0; q < f2; q++) {
            /* final partition id = q << b1 | p == the key's low `bits` bits */
            offs[(q << b1) | p] = o;
            o += h2[q];
        }
        base += h1[p];
    }
    free(tmp); free(h1); free(h2);
    return out;
}

/* bucket_chaining_join, hashing/joins/parallel_radix_join.cpp:291-354.
 * N = next_pow2(|R_i|), MASK = (N-1) << NUM_RADIX_BITS, chains via next[]/bucket[]
 * starting at 1; probe compares keys and counts (:339). */
static void bucket_chaining_join(const ora_tuple *Ri, uint64_t nr, const ora_tuple *Si, uint64_t ns,
                                 int bits, ora_result *res) {
    if (nr == 0 || ns == 0) return;
    uint64_t N = next_pow2(nr);
    uint32_t MASK = (uint32_t)((N - 1) << bits);
    int64_t *next = (int64_t *)malloc(sizeof(int64_t) * nr);
    int64_t *bucket = (int64_t *)calloc(N, sizeof(int64_t));
    for (uint64_t i = 0; i < nr;) {
        uint32_t idx = (Ri[i].key & MASK) >> bits;
        next[i] = bucket[idx];
        bucket[idx] = (int64_t)(++i);
    }
    for (uint64_t i = 0; i < ns; i++) {
        uint32_t idx = (Si[i].key & MASK) >> bits;
        for (int64_t hit = bucket[idx]; hit > 0; hit = next[hit - 1])
            if (Si[i].key == Ri[hit - 1].key) emit(res, Si[i].key, Ri[hit - 1].payload, Si[i].payload);
    }
    free(next); free(bucket);
}

/* histogram_join (PRH), hashing/joins/parallel_radix_join.cpp:373-432:
 * Nhist = max(4, next_pow2(|R_i|) >> 2) (get_hist_size :361-370), reorder R_i by
 * hist bucket, probe scans [hist[idx], hist[idx+1]). */
static void histogram_join(const ora_tuple *Ri, uint64_t nr, const ora_tuple *Si, uint64_t ns,
                           int bits, ora_result *res) {
    if (nr == 0 || ns == 0) return;
    uint64_t Nhist = next_pow2(nr) >> 2;
    if (Nhist < 4) Nhist = 4;
    uint32_t MASK = (uint32_t)((Nhist - 1) << bits);
    uint64_t *hist = (uint64_t *)calloc(Nhist + 2, sizeof(uint64_t));
    ora_tuple *tmp = (ora_tuple *)malloc(sizeof(ora_tuple) * nr);
    for (uint64_t i = 0; i < nr; i++) hist[((Ri[i].key & MASK) >> bits) + 2]++;
    for (uint64_t i = 2, sum = 0; i <= Nhist + 1; i++) { sum += hist[i]; hist[i] = sum; }
    for (uint64_t i = 0; i < nr; i++) {
        uint32_t idx = ((Ri[i].key & MASK) >> bits) + 1;
        tmp[hist[idx]++] = Ri[i];
    }
    for (uint64_t i = 0; i < ns; i++) {
        uint32_t idx = (Si[i].key & MASK) >> bits;
        for (uint64_t j = hist[idx]; j < hist[idx + 1]; j++)
            if (Si[i].key == tmp[j].key) emit(res, Si[i].key, tmp[j].payload, Si[i].payload);
    }
    free(hist); free(tmp);
}

static int radix_join(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS,
                      int bits, int histogram, ora_result *out) {
    if (!out || bits < 2 || bits > 24) return -1;
    memset(out, 0, sizeof(*out));
    uint32_t F = 1u << bits;
    uint64_t *offR = (uint64_t *)malloc(sizeof(uint64_t) * (F + 1));
    uint64_t *offS = (uint64_t *)malloc(sizeof(uint64_t) * (F + 1));
    ora_tuple *pR = two_pass_partition(R, nR, bits, offR);
    ora_tuple *pS = two_pass_partition(S, nS, bits, offS);
    /* partition sizes from the offsets of the pass-2 layout */
    uint64_t *cntR = (uint64_t *)calloc(F, sizeof(uint64_t));
    uint64_t *cntS = (uint64_t *)calloc(F, sizeof(uint64_t));
    for (uint64_t i = 0; i < nR; i++) cntR[R[i].key & (F - 1)]++;
    for (uint64_t i = 0; i < nS; i++) cntS[S[i].key & (F - 1)]++;
    /* join loop of prj_thread, :1409-1416 */
    for (uint32_t p = 0; p < F; p++) {
        if (histogram)
            histogram_join(pR + offR[p], cntR[p], pS + offS[p], cntS[p], bits, out);
        else
            bucket_chaining_join(pR + offR[p], cntR[p], pS + offS[p], cntS[p], bits, out);
    }
    free(offR); free(offS); free(pR); free(pS); free(cntR); free(cntS);
    return 0;
}

int ora_pro(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS, int bits, ora_result *out) {
    return radix_join(R, nR, S, nS, bits, 0, out);
}

int ora_prh(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS, int bits, ora_result *out) {
    return radix_join(R, nR, S, nS, bits, 1, out);
}

/* ------------------------------------------------------------------ */
/* NPO bucket hash table: hashing/joins/npj_types.h:32-38 (2 tuples +  */
/* overflow pointer), allocate_hashtable common_functions.cpp:75-102   */
/* (nbuckets = next_pow2(|R| / BUCKET_SIZE), no.._join.cpp:406-407),   */
/* HASH = key & (nb-1) (common_functions.h:57-58), build_hashtable_    */
/* single :172-206, probe_hashtable_single :237-280.                   */
/* ------------------------------------------------------------------ */
typedef struct ora_bucket {
    uint32_t count;
    ora_tuple tuples[2];
    struct ora_bucket *next;
} ora_bucket;

typedef struct { ora_bucket *buckets; uint64_t nb; uint32_t mask; } ora_ht;

static void ht_init(ora_ht *ht, uint64_t nbuckets) {
    ht->nb = next_pow2(nbuckets ? nbuckets : 1);
    ht->buckets = (ora_bucket *)calloc(ht->nb, sizeof(ora_bucket));
    ht->mask = (uint32_t)(ht->nb - 1);
}

static void ht_free(ora_ht *ht) {
    for (uint64_t i = 0; i < ht->nb; i++) {
        ora_bucket *b = ht->buckets[i].next;
        while (b) { ora_bucket *n = b->next; free(b); b = n; }
    }
    free(ht->buckets);
}

static void ht_insert(ora_ht *ht, ora_tuple t) {
    ora_bucket *curr = ht->buckets + (t.key & ht->mask);
    ora_bucket *nxt = curr->next;
    ora_tuple *dest;
    if (curr->count == 2) {
        if (!nxt || nxt->count == 2) {
            ora_bucket *b = (ora_bucket *)calloc(1, sizeof(ora_bucket));
            curr->next = b; b->next = nxt; b->count = 1; dest = b->tuples;
        } else {
            dest = nxt->tuples + nxt->count; nxt->count++;
        }
    } else {
        dest = curr->tuples + curr->count; curr->count++;
    }
    *dest = t;
}

/* probe with tuple t; `probe_is_r` says which side t is on */
static void ht_probe(const ora_ht *ht, ora_tuple t, int probe_is_r, ora_result *res) {
    const ora_bucket *b = ht->buckets + (t.key & ht->mask);
    do {
        for (uint32_t i = 0; i < b->count; i++)
            if (t.key == b->tuples[i].key) {
                if (probe_is_r) emit(res, t.key, t.payload, b->tuples[i].payload);
                else emit(res, t.key, b->tuples[i].payload, t.payload);
            }
        b = b->next;
    } while (b);
}

int ora_npo(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS, ora_result *out) {
    if (!out) return -1;
    memset(out, 0, sizeof(*out));
    ora_ht ht;
    ht_init(&ht, nR / 2);
    for (uint64_t i = 0; i < nR; i++) ht_insert(&ht, R[i]);      /* build_hashtable_mt :350-400 */
    for (uint64_t i = 0; i < nS; i++) ht_probe(&ht, S[i], 0, out); /* probe_hashtable :221-235 */
    ht_free(&ht);
    return 0;
}

/* SHJ: shj() hashing/helper/localjoiner.cpp:33-59 alternates one R and one S
 * tuple; SHJJoiner::join :73-94 inserts into its own side's table and probes
 * the other side's table (tables sized |R| and |S|, launcher.cpp:30-31). */
int ora_shj(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS, ora_result *out) {
    if (!out) return -1;
    memset(out, 0, sizeof(*out));
    ora_ht htR, htS;
    ht_init(&htR, nR / 2);
    ht_init(&htS, nS / 2);
    uint64_t iR = 0, iS = 0;
    while (iR < nR || iS < nS) {
        if (iR < nR) { ht_insert(&htR, R[iR]); ht_probe(&htS, R[iR], 1, out); iR++; }
        if (iS < nS) { ht_insert(&htS, S[iS]); ht_probe(&htR, S[iS], 0, out); iS++; }
    }
    ht_free(&htR); ht_free(&htS);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Sorting: tuples ordered as the 64-bit word key<<32 | payload, the   */
/* order of avxsort_tuples (sorting/joins/avxsort.cpp:209-223).        */
/* ------------------------------------------------------------------ */
static inline uint64_t word(ora_tuple t) { return ((uint64_t)t.key << 32) | t.payload; }

static void sort_tuples(ora_tuple *a, uint64_t n) {
    /* LSD radix sort, 4 x 16-bit digits of the 64-bit word */
    if (n < 2) return;
    ora_tuple *b = (ora_tuple *)malloc(sizeof(ora_tuple) * n);
    uint64_t *cnt = (uint64_t *)malloc(sizeof(uint64_t) * 65536);
    ora_tuple *src = a, *dst = b;
    for (int pass = 0; pass < 4; pass++) {
        int sh = 16 * pass;
        memset(cnt, 0, sizeof(uint64_t) * 65536);
        for (uint64_t i = 0; i < n; i++) cnt[(word(src[i]) >> sh) & 0xFFFF]++;
        uint64_t s = 0;
        for (int d = 0; d < 65536; d++) { uint64_t c = cnt[d]; cnt[d] = s; s += c; }
        for (uint64_t i = 0; i < n; i++) dst[cnt[(word(src[i]) >> sh) & 0xFFFF]++] = src[i];
        ora_tuple *t = src; src = dst; dst = t;
    }
    /* 4 passes: result is back in a */
    free(b); free(cnt);
}

/* merge_join, sorting/joins/common_functions.cpp:298-372, with the duplicate
 * cross-product of :318-351. */
static void merge_join(const ora_tuple *r, const ora_tuple *s, uint64_t nr, uint64_t ns, ora_result *res) {
    uint64_t i = 0, j = 0;
    while (i < nr && j < ns) {
        if (r[i].key < s[j].key) i++;
        else if (r[i].key > s[j].key) j++;
        else {
            uint64_t jj;
            do {
                jj = j;
                do {
                    emit(res, s[jj].key, r[i].payload, s[jj].payload);
                    jj++;
                } while (jj < ns && r[i].key == s[jj].key);
                i++;
            } while (i < nr && r[i].key == s[j].key);
            j = jj;
        }
    }
}

int ora_smj(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS, ora_result *out) {
    if (!out) return -1;
    memset(out, 0, sizeof(*out));
    ora_tuple *r = (ora_tuple *)malloc(sizeof(ora_tuple) * (nR ? nR : 1));
    ora_tuple *s = (ora_tuple *)malloc(sizeof(ora_tuple) * (nS ? nS : 1));
    memcpy(r, R, sizeof(ora_tuple) * nR);
    memcpy(s, S, sizeof(ora_tuple) * nS);
    /* partitioning_phase + sorting_phase + multiwaymerge_phase produce, per
     * thread, sorted runs over disjoint key ranges; one global sort gives the
     * same pairs (sortmergejoin_multiway.cpp:435-700). */
    sort_tuples(r, nR);
    sort_tuples(s, nS);
    merge_join(r, s, nR, nS, out);
    free(r); free(s);
    return 0;
}

/* ------------------------------------------------------------------ */
/* PMJ: PMJJoiner::join hashing/helper/localjoiner.cpp:512-600 buffers */
/* progressive_step tuples of each side, sorting_phase (pmj_helper.cpp */
/* :198-240) sorts the chunk pair and joins it (earlyJoinInitialRuns   */
/* :11-32, a sweep over both sorted chunks); merging_phase (:188-196,  */
/* earlyJoinMergedRuns :41-173) joins R of one run with S of every     */
/* OTHER run.                                                           */
/* ------------------------------------------------------------------ */
typedef struct { ora_tuple *r; uint64_t nr; ora_tuple *s; uint64_t ns; } ora_run;

/* earlyJoinInitialRuns: sweep areas RM/SM (pmj_helper.h:86-130); the sweep
 * drops entries with smaller keys and counts equal keys. */
static void early_join_initial(const ora_run *run, ora_result *res) {
    uint64_t r = 0, s = 0;
    /* the sweep areas hold the current equal-key group of each side */
    uint64_t rm_lo = 0, rm_hi = 0, sm_lo = 0, sm_hi = 0;
    while (r < run->nr || s < run->ns) {
        if (s == run->ns || (r < run->nr && run->r[r].key <= run->s[s].key)) {
            const ora_tuple *tr = &run->r[r];
            rm_hi = r + 1;                                   /* RM.insert(tr) */
            while (rm_lo < rm_hi && run->r[rm_lo].key < tr->key) rm_lo++;
            while (sm_lo < sm_hi && run->s[sm_lo].key < tr->key) sm_lo++; /* SM.query */
            for (uint64_t k = sm_lo; k < sm_hi; k++)
                if (run->s[k].key == tr->key) emit(res, tr->key, tr->payload, run->s[k].payload);
            r++;
        } else {
            const ora_tuple *ts = &run->s[s];
            sm_hi = s + 1;                                   /* SM.insert(ts) */
            while (sm_lo < sm_hi && run->s[sm_lo].key < ts->key) sm_lo++;
            while (rm_lo < rm_hi && run->r[rm_lo].key < ts->key) rm_lo++; /* RM.query */
            for (uint64_t k = rm_lo; k < rm_hi; k++)
                if (run->r[k].key == ts->key) emit(res, ts->key, run->r[k].payload, ts->payload);
            s++;
        }
    }
}

int ora_pmj(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS,
            uint64_t step_r, uint64_t step_s, ora_result *out) {
    if (!out) return -1;
    memset(out, 0, sizeof(*out));
    if (step_r == 0) step_r = 1;
    if (step_s == 0) step_s = 1;
    uint64_t nruns_r = (nR + step_r - 1) / step_r, nruns_s = (nS + step_s - 1) / step_s;
    uint64_t nruns = nruns_r > nruns_s ? nruns_r : nruns_s;
    if (nruns == 0) return 0;
    ora_run *runs = (ora_run *)calloc(nruns, sizeof(ora_run));
    for (uint64_t k = 0; k < nruns; k++) {
        uint64_t r0 = k * step_r, s0 = k * step_s;
        /* the last run takes the left-over of both sides (localjoiner.cpp:575-590) */
        uint64_t r1 = (k + 1 == nruns) ? nR : (r0 + step_r < nR ? r0 + step_r : nR);
        uint64_t s1 = (k + 1 == nruns) ? nS : (s0 + step_s < nS ? s0 + step_s : nS);
        if (r0 > nR) r0 = nR;
        if (s0 > nS) s0 = nS;
        runs[k].nr = r1 - r0; runs[k].ns = s1 - s0;
        runs[k].r = (ora_tuple *)malloc(sizeof(ora_tuple) * (runs[k].nr + 1));
        runs[k].s = (ora_tuple *)malloc(sizeof(ora_tuple) * (runs[k].ns + 1));
        memcpy(runs[k].r, R + r0, sizeof(ora_tuple) * runs[k].nr);
        memcpy(runs[k].s, S + s0, sizeof(ora_tuple) * runs[k].ns);
        sort_tuples(runs[k].r, runs[k].nr);
        sort_tuples(runs[k].s, runs[k].ns);
        early_join_initial(&runs[k], out);
    }
    /* merging phase: R of run i with S of run j, i != j */
    for (uint64_t i = 0; i < nruns; i++)
        for (uint64_t j = 0; j < nruns; j++)
            if (i != j) merge_join(runs[i].r, runs[j].s, runs[i].nr, runs[j].ns, out);
    for (uint64_t k = 0; k < nruns; k++) { free(runs[k].r); free(runs[k].s); }
    free(runs);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Independent truth (no reference structure): sort, group equal keys, */
/* enumerate the cross product of each group pair.                     */
/* ------------------------------------------------------------------ */
int ora_truth(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS, ora_result *out) {
    if (!out) return -1;
    memset(out, 0, sizeof(*out));
    ora_tuple *r = (ora_tuple *)malloc(sizeof(ora_tuple) * (nR ? nR : 1));
    ora_tuple *s = (ora_tuple *)malloc(sizeof(ora_tuple) * (nS ? nS : 1));
    memcpy(r, R, sizeof(ora_tuple) * nR);
    memcpy(s, S, sizeof(ora_tuple) * nS);
    sort_tuples(r, nR);
    sort_tuples(s, nS);
    uint64_t i = 0, j = 0;
    while (i < nR && j < nS) {
        uint32_t kr = r[i].key, ks = s[j].key;
        if (kr < ks) { i++; continue; }
        if (kr > ks) { j++; continue; }
        uint64_t ie = i, je = j;
        while (ie < nR && r[ie].key == kr) ie++;
        while (je < nS && s[je].key == kr) je++;
        for (uint64_t a = i; a < ie; a++)
            for (uint64_t b = j; b < je; b++) emit(out, kr, r[a].payload, s[b].payload);
        i = ie; j = je;
    }
    free(r); free(s);
    return 0;
}

uint64_t ora_materialize_sorted(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS,
                                ora_tuple *out, uint64_t cap) {
    ora_tuple *r = (ora_tuple *)malloc(sizeof(ora_tuple) * (nR ? nR : 1));
    ora_tuple *s = (ora_tuple *)malloc(sizeof(ora_tuple) * (nS ? nS : 1));
    memcpy(r, R, sizeof(ora_tuple) * nR);
    memcpy(s, S, sizeof(ora_tuple) * nS);
    sort_tuples(r, nR);
    sort_tuples(s, nS);
    uint64_t i = 0, j = 0, n = 0;
    while (i < nR && j < nS) {
        uint32_t kr = r[i].key, ks = s[j].key;
        if (kr < ks) { i++; continue; }
        if (kr > ks) { j++; continue; }
        uint64_t ie = i, je = j;
        while (ie < nR && r[ie].key == kr) ie++;
        while (je < nS && s[je].key == kr) je++;
        for (uint64_t a = i; a < ie; a++)
            for (uint64_t b = j; b < je; b++) {
                if (n < cap) out[n] = s[b];   /* <S-key, S-payload> */
                n++;
            }
        i = ie; j = je;
    }
    if (n <= cap) sort_tuples(out, n);
    free(r); free(s);
    return n;
}

/* ------------------------------------------------------------------ */
/* Direct-address truth for a build side with unique keys (the PK side */
/* of every foreign-key configuration).  payload_of[key] and a         */
/* presence bit per key are filled from R, then each S tuple looks up  */
/* its key: no partitioning, hashing or sorting, so it shares nothing  */
/* with the restatements above and stays cheap at 2^27 tuples.         */
/* ------------------------------------------------------------------ */
int ora_pk_truth(const ora_tuple *R, uint64_t nR, const ora_tuple *S, uint64_t nS, ora_result *out) {
    out->count = 0;
    out->checksum = 0;
    uint64_t maxkey = 0;
    for (uint64_t i = 0; i < nR; i++)
        if (R[i].key > maxkey) maxkey = R[i].key;
    if (maxkey > 8 * nR + (1u << 20)) return -2;   /* keys not dense enough for a direct table */
    const uint64_t slots = maxkey + 1;
    uint32_t *payload_of = (uint32_t *)malloc(sizeof(uint32_t) * slots);
    uint64_t *present = (uint64_t *)calloc((slots + 63) / 64, sizeof(uint64_t));
    if (!payload_of || !present) { free(payload_of); free(present); return -3; }
    for (uint64_t i = 0; i < nR; i++) {
        if (i + 16 < nR && R[i + 16].key <= maxkey) {
            __builtin_prefetch(&payload_of[R[i + 16].key], 1);
            __builtin_prefetch(&present[R[i + 16].key >> 6], 1);
        }
        const uint32_t k = R[i].key;
        const uint64_t bit = 1ull << (k & 63);
        if (present[k >> 6] & bit) { free(payload_of); free(present); return -1; }   /* repeated key */
        present[k >> 6] |= bit;
        payload_of[k] = R[i].payload;
    }
    for (uint64_t j = 0; j < nS; j++) {
        if (j + 16 < nS && S[j + 16].key <= maxkey) {   /* random lookups: keep several in flight */
            __builtin_prefetch(&payload_of[S[j + 16].key]);
            __builtin_prefetch(&present[S[j + 16].key >> 6]);
        }
        const uint32_t k = S[j].key;
        if (k <= maxkey && (present[k >> 6] >> (k & 63)) & 1) emit(out, k, payload_of[k], S[j].payload);
    }
    free(payload_of);
    free(present);
    return 0;
}
