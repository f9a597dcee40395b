/*
 * qphix_d3_generic.h -- generic names mapped to the double-precision API when
 * QPHIX_Precision == 'D'; replaces the reference qphix_d3_generic.h
 * (same mapping, so MILC's generic calls resolve identically).
 */
#ifndef _QPHIX_D3__PC_GENERIC_H
#define _QPHIX_D3__PC_GENERIC_H

#define QPHIX_asqtad_create_L_from_raw QPHIX_D3_asqtad_create_L_from_raw
#define QPHIX_asqtad_destroy_L QPHIX_D3_asqtad_destroy_L
#define QPHIX_asqtad_invert_multi QPHIX_D3_asqtad_invert_multi
#define QPHIX_asqtad_invert QPHIX_D3_asqtad_invert
#define QPHIX_create_V_from_raw QPHIX_D3_create_V_from_raw
#define QPHIX_create_G_from_raw QPHIX_D3_create_G_from_raw
#define QPHIX_create_F_from_raw QPHIX_D3_create_F_from_raw
#define QPHIX_destroy_V QPHIX_D3_destroy_V
#define QPHIX_destroy_G QPHIX_D3_destroy_G
#define QPHIX_destroy_F QPHIX_D3_destroy_F
#define QPHIX_extract_V_to_raw QPHIX_D3_extract_V_to_raw
#define QPHIX_extract_G_to_raw QPHIX_D3_extract_G_to_raw
#define QPHIX_extract_F_to_raw QPHIX_D3_extract_F_to_raw
#define QPHIX_symanzik_1loop_gauge_force QPHIX_D3_symanzik_1loop_gauge_force
#define QPHIX_ColorVector QPHIX_D3_ColorVector
#define QPHIX_FermionLinksAsqtad QPHIX_D3_FermionLinksAsqtad
#define QPHIX_Force QPHIX_D3_Force
#define QPHIX_GaugeField QPHIX_D3_GaugeField

#endif
