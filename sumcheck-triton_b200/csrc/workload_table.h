// GENERATED by gen_workload_table.py from zkduel_b200.workloads -- do not edit by hand.
// The 32 kernel workloads: name, polynomial, id, tables, degree, terms, and where their
// terms start in kTermCoeffs / kTermLens and their factors (kernel table indices) in kFlat.
#pragma once
#include <cstdint>

namespace sc_cli {

struct WorkloadDef {
  const char* name;
  const char* poly;
  int id, vars, degree, terms;
  int term0, flat0;
};

constexpr int kNumWorkloads = 32;
constexpr WorkloadDef kWorkloads[] = {
    {"poly_a", "a", 1, 1, 1, 1, 0, 0},
    {"poly_ab", "a*b", 2, 2, 2, 1, 1, 1},
    {"poly_ab_plus_c", "a*b + c", 3, 3, 2, 2, 2, 3},
    {"poly_abc", "a*b*c", 4, 3, 3, 1, 4, 6},
    {"poly_aabbc", "a*a*b*b*c", 5, 3, 5, 1, 5, 9},
    {"poly_abc_plus_de", "a*b*c + d*e", 6, 5, 3, 2, 6, 14},
    {"poly_abcg_plus_deg", "a*b*c*g + d*e*g", 7, 6, 4, 2, 8, 19},
    {"zk_verifiable_asics", "qadd*a + qadd*b + qmul*a*b", 8, 4, 3, 3, 10, 26},
    {"zk_spartan_1", "A*B*fz - C*fz", 9, 4, 3, 2, 13, 33},
    {"zk_spartan_2", "ABC*Z", 10, 2, 2, 1, 15, 38},
    {"zk_witness_non_id", "q_non-id-point*y*y - q_non-id-point*x*x*x - 5*q_non-id-point", 11, 3, 4, 3, 16, 40},
    {"zk_complete_add_1", "q_add*x_q*x_q*lambda - 2*q_add*x_q*x_p*lambda + q_add*x_p*x_p*lambda - q_add*x_q*y_q + q_add*x_q*y_p + q_add*x_p*y_q - q_add*x_p*y_p", 12, 6, 4, 7, 19, 48},
    {"zk_complete_add_7", "q_add*x_r - q_add*x_q - q_add*x_p*x_r*beta + q_add*x_p*x_q*beta", 13, 5, 4, 4, 26, 72},
    {"zk_complete_add_8", "q_add*y_r - q_add*y_q - q_add*x_p*y_r*beta + q_add*x_p*y_q*beta", 14, 5, 4, 4, 30, 84},
    {"zk_witness_id_point_1", "q_point*x*y*y - q_point*x*x*x*x - 5*q_point*x", 15, 3, 5, 3, 34, 96},
    {"zk_witness_id_point_2", "q_point*y*y*y - q_point*y*x*x*x - 5*q_point*y", 16, 3, 5, 3, 37, 107},
    {"zk_incomplete_add_1", "q_add-incomplete*x_r*x_p*x_p - 2*q_add-incomplete*x_r*x_p*x_q + q_add-incomplete*x_r*x_q*x_q + q_add-incomplete*x_q*x_p*x_p - 2*q_add-incomplete*x_q*x_q*x_p + q_add-incomplete*x_q*x_q*x_q + q_add-incomplete*x_p*x_p*x_p - 2*q_add-incomplete*x_p*x_p*x_q + q_add-incomplete*x_p*x_q*x_q - q_add-incomplete*y_p*y_p + 2*q_add-incomplete*y_p*y_q - q_add-incomplete*y_q*y_q", 17, 6, 4, 12, 40, 118},
    {"zk_incomplete_add_2", "q_add-incomplete*y_r*x_p - q_add-incomplete*y_r*x_q + q_add-incomplete*y_q*x_p - q_add-incomplete*y_q*x_q - q_add-incomplete*y_p*x_q + q_add-incomplete*y_p*x_r - q_add-incomplete*y_q*x_r + q_add-incomplete*y_q*x_q", 18, 7, 3, 8, 52, 163},
    {"zk_complete_add_2", "2*q_add*y_p*lambda - 3*q_add*x_p*x_p - 2*q_add*x_q*y_p*lambda*alpha + 3*q_add*x_q*x_p*x_p*alpha + 2*q_add*x_p*y_p*lambda*alpha - 3*q_add*x_p*x_p*x_p*alpha", 19, 6, 5, 6, 60, 187},
    {"zk_complete_add_3", "q_add*x_p*x_q*x_q*lambda*lambda - q_add*x_p*x_q*x_q*x_q - q_add*x_p*x_q*x_q*x_r - q_add*x_p*x_p*x_q*x_q - q_add*x_p*x_p*x_q*lambda*lambda + q_add*x_p*x_p*x_p*x_q + q_add*x_p*x_p*x_q*x_r + q_add*x_p*x_p*x_q*x_q", 20, 5, 6, 8, 66, 213},
    {"zk_complete_add_4", "q_add*x_p*x_p*x_q*x_q*lambda - q_add*x_p*x_q*x_q*x_r*lambda - q_add*x_p*x_q*x_q*y_p - q_add*x_p*x_q*x_q*y_r - q_add*x_p*x_p*x_p*x_q*lambda + q_add*x_p*x_p*x_q*x_r*lambda + q_add*x_p*x_p*x_q*y_p + q_add*x_p*x_p*x_q*y_r", 21, 7, 6, 8, 74, 255},
    {"zk_complete_add_5", "q_add*x_p*x_q*y_q*lambda*lambda + q_add*x_p*x_q*y_p*lambda*lambda - q_add*x_p*x_p*x_q*y_q - q_add*x_p*x_p*x_q*y_p - q_add*x_p*x_q*x_q*y_q - q_add*x_p*x_q*x_q*y_p - q_add*x_p*x_q*y_q*x_r - q_add*x_p*x_q*y_p*x_r", 22, 7, 6, 8, 82, 299},
    {"zk_complete_add_6", "q_add*x_p*x_p*x_q*y_q*lambda + q_add*x_p*x_p*x_q*y_p*lambda - q_add*x_p*x_q*y_p*x_r*lambda - q_add*x_p*x_q*y_q*x_r*lambda - q_add*x_p*x_q*y_p*y_p - q_add*x_p*x_q*y_p*y_q - q_add*x_p*x_q*y_p*y_r - q_add*x_p*x_q*y_q*y_r", 23, 8, 6, 8, 90, 341},
    {"zk_complete_add_9", "q_add*x_r - q_add*x_p - q_add*x_q*x_r*gamma + q_add*x_p*x_q*gamma", 24, 5, 4, 4, 98, 385},
    {"zk_complete_add_10", "q_add*y_r - q_add*y_p - q_add*x_q*y_r*gamma + q_add*x_q*y_p*gamma", 25, 5, 4, 4, 102, 397},
    {"zk_complete_add_11", "q_add*x_r - q_add*x_q*x_r*alpha + q_add*x_p*x_r*alpha - q_add*y_q*x_r*delta - q_add*y_p*x_r*delta", 26, 8, 4, 5, 106, 409},
    {"zk_complete_add_12", "q_add*y_r - q_add*x_q*y_r*alpha + q_add*x_p*y_r*alpha - q_add*y_q*y_r*delta - q_add*y_p*y_r*delta", 27, 8, 4, 5, 111, 427},
    {"zk_vanilla_zerocheck_hp", "qL*w1*fz1 + qR*w2*fz1 + qM*w1*w2*fz1 - qO*w3*fz1 + qC*fz1", 28, 9, 4, 5, 116, 445},
    {"zk_vanilla_permcheck_hp", "pi*fz2 - p1*p2*fz2 + 7*phi*D1*D2*D3*fz2 - 7*N1*N2*N3*fz2", 29, 11, 5, 4, 121, 460},
    {"zk_jellyfish_zerocheck_hp", "qL*w1*fz + qR*w2*fz + qM*w1*w2*fz - qO*w3*fz + q1*w1*fz + q2*w2*fz + q3*w3*fz + q4*w4*fz - qO*w5*fz + qM1*w1*w2*fz + qM2*w3*w4*fz + qH1*w1*w1*w1*w1*w1*fz + qH2*w2*w2*w2*w2*w2*fz + qH3*w3*w3*w3*w3*w3*fz + qH4*w4*w4*w4*w4*w4*fz + qECC*w1*w2*w3*w4*fz + qc*fz", 30, 22, 7, 17, 125, 474},
    {"zk_jellyfish_permcheck_hp", "pi*fz - p1*p2*fz + 7*phi*D1*D2*D3*D4*D5*fz - 7*N1*N2*N3*N4*N5*fz", 31, 15, 7, 4, 142, 546},
    {"zk_opencheck", "y1*k1 + y2*k2 + y3*k3 + y4*k4 + y5*k5 + y6*k6", 32, 12, 2, 6, 146, 564},
};
constexpr int64_t kTermCoeffs[] = {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, 1, 1, -1, -5, 1, -2, 1, -1, 1, 1, -1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -5, 1, -1, -5, 1, -2, 1, 1, -2, 1, 1, -2, 1, -1, 2, -1, 1, -1, 1, -1, -1, 1, -1, 1, 2, -3, -2, 3, 2, -3, 1, -1, -1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, -1, 1, 1, -1, -1, -1, -1, -1, -1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1, -1, 1, -1, 1, -1, -1, 1, 1, 1, -1, 1, 1, -1, 7, -7, 1, 1, 1, -1, 1, 1, 1, 1, -1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, 7, -7, 1, 1, 1, 1, 1, 1};
constexpr int32_t kTermLens[] = {1, 2, 2, 1, 3, 5, 3, 2, 4, 3, 2, 2, 3, 3, 2, 2, 3, 4, 1, 4, 4, 4, 3, 3, 3, 3, 2, 2, 4, 4, 2, 2, 4, 4, 4, 5, 2, 4, 5, 2, 4, 4, 4, 4, 4, 4, 4, 4, 4, 3, 3, 3, 3, 3, 3, 3, 3, 3, 3, 3, 3, 3, 5, 5, 5, 5, 6, 5, 5, 5, 6, 5, 5, 5, 6, 6, 5, 5, 6, 6, 5, 5, 6, 6, 5, 5, 5, 5, 5, 5, 6, 6, 6, 6, 5, 5, 5, 5, 2, 2, 4, 4, 2, 2, 4, 4, 2, 4, 4, 4, 4, 2, 4, 4, 4, 4, 3, 3, 4, 3, 2, 2, 3, 5, 4, 3, 3, 4, 3, 3, 3, 3, 3, 3, 4, 4, 7, 7, 7, 7, 6, 2, 2, 3, 7, 6, 2, 2, 2, 2, 2, 2};
constexpr int32_t kFlat[] = {0, 0, 1, 0, 1, 2, 0, 1, 2, 0, 0, 1, 1, 2, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 5, 3, 0, 1, 0, 2, 3, 1, 2, 0, 1, 2, 3, 2, 0, 1, 0, 1, 1, 0, 2, 2, 2, 0, 0, 1, 1, 3, 0, 1, 2, 3, 0, 2, 2, 3, 0, 1, 4, 0, 1, 5, 0, 2, 4, 0, 2, 5, 0, 1, 0, 2, 0, 3, 1, 4, 0, 3, 2, 4, 0, 1, 0, 2, 0, 3, 1, 4, 0, 3, 2, 4, 0, 1, 2, 2, 0, 1, 1, 1, 1, 0, 1, 0, 1, 1, 1, 0, 1, 2, 2, 2, 0, 1, 0, 1, 2, 2, 0, 1, 2, 3, 0, 1, 3, 3, 0, 3, 2, 2, 0, 3, 3, 2, 0, 3, 3, 3, 0, 2, 2, 2, 0, 2, 2, 3, 0, 2, 3, 3, 0, 4, 4, 0, 4, 5, 0, 5, 5, 0, 1, 2, 0, 1, 3, 0, 4, 2, 0, 4, 3, 0, 5, 3, 0, 5, 6, 0, 4, 6, 0, 4, 3, 0, 1, 2, 0, 3, 3, 0, 4, 1, 2, 5, 0, 4, 3, 3, 5, 0, 3, 1, 2, 5, 0, 3, 3, 3, 5, 0, 1, 2, 2, 3, 3, 0, 1, 2, 2, 2, 0, 1, 2, 2, 4, 0, 1, 1, 2, 2, 0, 1, 1, 2, 3, 3, 0, 1, 1, 1, 2, 0, 1, 1, 2, 4, 0, 1, 1, 2, 2, 0, 1, 1, 2, 2, 3, 0, 1, 2, 2, 4, 3, 0, 1, 2, 2, 5, 0, 1, 2, 2, 6, 0, 1, 1, 1, 2, 3, 0, 1, 1, 2, 4, 3, 0, 1, 1, 2, 5, 0, 1, 1, 2, 6, 0, 1, 2, 3, 4, 4, 0, 1, 2, 5, 4, 4, 0, 1, 1, 2, 3, 0, 1, 1, 2, 5, 0, 1, 2, 2, 3, 0, 1, 2, 2, 5, 0, 1, 2, 3, 6, 0, 1, 2, 5, 6, 0, 1, 1, 2, 3, 4, 0, 1, 1, 2, 5, 4, 0, 1, 2, 5, 6, 4, 0, 1, 2, 3, 6, 4, 0, 1, 2, 5, 5, 0, 1, 2, 5, 3, 0, 1, 2, 5, 7, 0, 1, 2, 3, 7, 0, 1, 0, 2, 0, 3, 1, 4, 0, 2, 3, 4, 0, 1, 0, 2, 0, 3, 1, 4, 0, 3, 2, 4, 0, 1, 0, 2, 1, 3, 0, 4, 1, 3, 0, 5, 1, 6, 0, 7, 1, 6, 0, 1, 0, 2, 1, 3, 0, 4, 1, 3, 0, 5, 1, 6, 0, 7, 1, 6, 0, 1, 2, 3, 4, 2, 5, 1, 4, 2, 6, 7, 2, 8, 2, 0, 1, 2, 3, 1, 4, 5, 6, 7, 1, 8, 9, 10, 1, 0, 1, 2, 3, 4, 2, 5, 1, 4, 2, 6, 7, 2, 8, 1, 2, 9, 4, 2, 10, 7, 2, 11, 12, 2, 6, 13, 2, 14, 1, 4, 2, 15, 7, 12, 2, 16, 1, 1, 1, 1, 1, 2, 17, 4, 4, 4, 4, 4, 2, 18, 7, 7, 7, 7, 7, 2, 19, 12, 12, 12, 12, 12, 2, 20, 1, 4, 7, 12, 2, 21, 2, 0, 1, 2, 3, 1, 4, 5, 6, 7, 8, 9, 1, 10, 11, 12, 13, 14, 1, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11};

// The four fields (zkduel_b200.fields.FIELD_SPECS): name, bit width, limbs, -p^-1 mod 2^32,
// modulus in hex, little-endian modulus limbs.
struct FieldDef {
  const char* name;
  int bit_width, limbs;
  uint32_t nprime;
  const char* modulus_hex;
  uint32_t modulus[8];
};
constexpr int kNumFields = 4;
constexpr FieldDef kFields[] = {
    {"p32_2^32_minus_5", 32, 1, 0xcccccccdu, "0xfffffffb", {0xfffffffbu}},
    {"p64_goldilocks", 64, 2, 0xffffffffu, "0xffffffff00000001", {0x00000001u, 0xffffffffu}},
    {"p128_mersenne_2^127_minus_1", 128, 4, 0x00000001u, "0x7fffffffffffffffffffffffffffffff", {0xffffffffu, 0xffffffffu, 0xffffffffu, 0x7fffffffu}},
    {"p255_bls12_381_scalar", 256, 8, 0xffffffffu, "0x73eda753299d7d483339d80809a1d80553bda402fffe5bfeffffffff00000001", {0x00000001u, 0xffffffffu, 0xfffe5bfeu, 0x53bda402u, 0x09a1d805u, 0x3339d808u, 0x299d7d48u, 0x73eda753u}},
};

}  // namespace sc_cli
