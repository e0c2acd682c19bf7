void pe_oracle_placeholder(void){}
